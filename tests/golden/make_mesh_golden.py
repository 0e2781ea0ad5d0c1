"""Generate tests/golden/mesh_*.npz: the reference's own mesh build of the
flow task (BaseTaskDescription::buildMesh, base_task_description.h:330-371:
level set, calcAlpha with its oscillation fix, calcTypeOfCells, calcTheta,
buildCV_U/V/W, buildMeshFunctions, buildDelta_ib, buildInvBaseDelta_ib) on
uniform grids with level-set bodies, dumped by the harness's mesh_dump mode
(oracle/_ref/ref_harness, built by oracle/build_ref.sh).  Run from the
repository root:

    python tests/golden/make_mesh_golden.py

Cases: one sphere off the grid lines (16^3), one sphere centred on a cell
corner so that its poles put phi = 0 exactly on corners (16^3, the
degenerate case the reference's own sphere task avoids by a half-cell shift),
a flat box 20x12x10, four seeded spheres (24^3), three seeded rotated
ellipsoids (64x32x32), two spheres cutting the bottom and top walls
(16x16x12), and the 128x64x64 sphere flow box.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "ls-stag-3d_parallel_b200"))

import ref_runner as rr  # noqa: E402
from lsstag_b200 import synth  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))

KEEP = ["dims", "ls_block", "h", "phi_ls", "phi", "alpha", "side_type", "celltype", "theta", "delta", "nodes", "vof",
        "inv_vof", "xtype", "ytype", "ztype", "vof_x", "vof_y", "vof_z", "inv_mx", "inv_my", "inv_mz", "dib_en",
        "dib_ws", "dib_nb", "dib_st", "dib_max", "inv_dib_ne", "inv_dib_tn"]


def cases():
    out = []
    h = 1.0 / 16
    out.append(("sphere16", rr.Case(16, 16, 16, h, h, h, spheres=[(0.5 + 0.3 * h, 0.5 + 0.2 * h, 0.5 + 0.1 * h, 0.18)])))
    out.append(("sphere16_vertex", rr.Case(16, 16, 16, h, h, h, spheres=[(0.5, 0.5, 0.5, 0.25)])))
    h = 1.0 / 20
    out.append(("sphere20x12x10", rr.Case(20, 12, 10, h, h, h,
                                          spheres=[(0.5 + 0.3 * h, 0.3 + 0.2 * h, 0.25 + 0.1 * h, 0.09)])))
    h = 1.0 / 24
    out.append(("spheres4_24", rr.Case(24, 24, 24, h, h, h,
                                       spheres=synth.four_spheres(3, rmin=0.05, rmax=0.1, cmin=0.4, cmax=0.6))))
    # the large-flow generator's bodies (semi-axes U[0.3, 0.8], random
    # rotations, centres in the first third), moved 1 along x so that the
    # level-set block stays 5 cells clear of the inflow wall at h = 1/8
    h = 1.0 / 8
    ell = synth.ellipsoids(5, 3, (8.0, 4.0, 4.0), amin=0.3, amax=0.8)
    ell = [(np.asarray(c, float) + np.array([1.0, 0.0, 0.0]), a, rot) for (c, a, rot) in ell]
    out.append(("ellipsoids3_64x32x32", rr.Case(64, 32, 32, h, h, h, ellipsoids=ell)))
    # spheres cutting the bottom and top walls: the first and last layers'
    # own walks (bottom- / topBuildAlpha, bottom- / topTypeOfCell,
    # tbBuildTheta) and the border cells' face-shape cases
    h = 1.0 / 16
    out.append(("walls16x16x12", rr.Case(16, 16, 12, h, h, h, spheres=[(0.5 + 0.01, 0.5 - 0.02, 0.03, 0.15),
                                                                        (0.47, 0.52, 0.74, 0.14)])))
    out.append(("flow_sphere_128x64x64", rr.Case(128, 64, 64, h, h, h,
                                                 spheres=[(2.0, 2.0 + 0.5 * h, 2.0 + 0.5 * h, 0.5)])))
    return out


def main():
    if not rr.available():
        sys.exit("oracle/_ref/ref_harness missing: run oracle/build_ref.sh first")
    for name, case in cases():
        r = rr.run(case, threads=1, mesh_dump=1, timeout=3000)
        keep = {k: r[k] for k in KEEP}
        keep["spheres"] = np.array(case.spheres, dtype=np.float64).reshape(-1, 4)
        ell = [np.concatenate([np.asarray(c, float), np.asarray(a, float), np.asarray(rot, float).reshape(-1)])
               for (c, a, rot) in case.ellipsoids]
        keep["ellipsoids"] = np.array(ell, dtype=np.float64).reshape(-1, 15)
        path = os.path.join(HERE, f"mesh_{name}.npz")
        np.savez_compressed(path, **keep)
        print(f"{path}: dims={tuple(int(v) for v in r['dims'])} block={r['ls_block'].tolist()} "
              f"cut={int(np.sum((r['celltype'] > 0) & (r['celltype'] < 11111111)))} size={os.path.getsize(path)} B")


if __name__ == "__main__":
    main()
