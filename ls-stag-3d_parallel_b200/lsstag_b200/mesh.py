"""The flow task's mesh build on the device: the counterpart of the
reference's LSSTAGUniformMesh build for a flow past fixed bodies on a uniform
grid (BaseTaskDescription::buildMesh, base_task_description.h:330-371), run by
lsg_mesh_build.  The arrays it produces (cell and face types, edge and face
fractions, cell volumes, staggered types and inverse volumes) are the
reference's, bit for bit, and stay on the device: IterativeSolver.set_from_mesh
assembles the pressure operator from them without a host round trip.

Bodies are given as records of 17 doubles (``sphere``, ``ellipsoid``); the
level-set block is the task's (``flow_block``).
"""
from __future__ import annotations

import math

import numpy as np

BODY_WORDS = 17

# name -> (field code, dtype, grid): grid "n" base cells, "3n" coord triples,
# "x" / "y" / "z" the staggered grids
FIELDS = {
    "phi_ls": (0, np.float64, "n"), "phi": (1, np.float64, "n"), "alpha": (2, np.float64, "3n"),
    "side_type": (3, np.int32, "3n"), "celltype": (4, np.int32, "n"), "theta": (5, np.float64, "3n"),
    "delta": (6, np.float64, "3n"), "vof": (7, np.float64, "n"), "inv_vof": (8, np.float64, "n"),
    "xtype": (9, np.int32, "x"), "ytype": (10, np.int32, "y"), "ztype": (11, np.int32, "z"),
    "vof_x": (12, np.float64, "x"), "vof_y": (13, np.float64, "y"), "vof_z": (14, np.float64, "z"),
    "inv_mx": (15, np.float64, "x"), "inv_my": (16, np.float64, "y"), "inv_mz": (17, np.float64, "z"),
    "dib_en": (18, np.float64, "3n"), "dib_ws": (19, np.float64, "3n"), "dib_nb": (20, np.float64, "3n"),
    "dib_st": (21, np.float64, "3n"), "dib_max": (22, np.float64, "3n"), "inv_dib_ne": (23, np.float64, "3n"),
    "inv_dib_tn": (24, np.float64, "3n"),
}


def sphere(center, radius) -> np.ndarray:
    """Body record of a sphere (phi = r - |x - c|, calcLevelSetSphere)."""
    rec = np.zeros(BODY_WORDS)
    rec[0] = 0.0
    rec[1:4] = center
    rec[4] = radius
    return rec


def ellipsoid(center, axes, rotation) -> np.ndarray:
    """Body record of an ellipsoid with semi-axes ``axes`` in the body frame
    R (x - c), R = ``rotation`` (3x3)."""
    rec = np.zeros(BODY_WORDS)
    rec[0] = 1.0
    rec[1:4] = center
    rec[5:8] = axes
    rec[8:17] = np.asarray(rotation, dtype=np.float64).reshape(9)
    return rec


def bodies_array(spheres=(), ellipsoids=()) -> np.ndarray:
    """Records of (cx, cy, cz, r) spheres and (c, axes, rotation) ellipsoids."""
    recs = [sphere(s[:3], s[3]) for s in spheres] + [ellipsoid(c, a, r) for (c, a, r) in ellipsoids]
    return np.ascontiguousarray(np.array(recs, dtype=np.float64).reshape(-1, BODY_WORDS))


def flow_block(dims, h, spheres=(), ellipsoids=()):
    """The level-set block (hs, hf, vs, vf) of a flow task over these bodies,
    as the uniform-grid flow task sets it: the bodies' bounding box in cells
    (hs = floor(lo / h), hf = floor(hi / h) + 1, as
    FlowSphereTaskDescription::initMeshParams takes xCellIndex(P_C.x - rad)
    and xCellIndex(P_C.x + rad) + 1, flow_sphere_task_description.h:126-137),
    kept at least 5 cells off the walls (the reference's sphere task keeps
    2; the uniform-grid cases here keep 5 so that the widened block below
    leaves 2 plain cells at every wall), then widened by 3 cells on each side
    (FlowTaskDescription::buildBaseMesh, flow_task_description.h:388-398)."""
    N, M, _ = (int(v) for v in dims)
    lo = [math.inf] * 3
    hi = [-math.inf] * 3
    for (cx, cy, cz, r) in spheres:
        for d, c in enumerate((cx, cy, cz)):
            lo[d] = min(lo[d], c - r)
            hi[d] = max(hi[d], c + r)
    for (c, a, _rot) in ellipsoids:
        e = float(np.max(a))
        for d in range(3):
            lo[d] = min(lo[d], float(c[d]) - e)
            hi[d] = max(hi[d], float(c[d]) + e)
    hs = max(5, math.floor(lo[0] / h[0]))
    hf = min(N - 5, math.floor(hi[0] / h[0]) + 1)
    vs = max(5, math.floor(lo[1] / h[1]))
    vf = min(M - 5, math.floor(hi[1] / h[1]) + 1)
    return (hs - 3, hf + 3, vs - 3, vf + 3)


def field_size(name: str, dims) -> int:
    N, M, K = (int(v) for v in dims)
    grid = FIELDS[name][2]
    return {"n": N * M * K, "3n": 3 * N * M * K, "x": (N - 1) * M * K, "y": N * (M - 1) * K,
            "z": N * M * (K - 1)}[grid]
