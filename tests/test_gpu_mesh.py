"""The flow task's mesh build on the GPU (lsg_mesh_build) against the
reference's own mesh build, array by array and bit for bit
(tests/golden/mesh_*.npz, dumped by the reference harness's mesh_dump mode:
level set as evaluated and after the oscillation fix, alpha, face and cell
types, theta, cell volumes and their inverses, staggered types, volumes and
inverse volumes, immersed-boundary face areas and inverse distances).
Cases: spheres off and on the grid lines (a pole on a cell corner), four
spheres, three rotated ellipsoids, two spheres cutting the bottom and top
walls, the 128x64x64 flow box; together they reach all 106 volume formulas,
the border cells' face shapes and oscillation-fix chains of up to three
cells.  Then the pressure operator assembled from the device mesh
(lsg_set_matrix_mesh) against the reference's own CSR."""
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

CASES = sorted(glob.glob(os.path.join(GOLDEN, "mesh_*.npz")))
FIELDS = ["phi_ls", "phi", "alpha", "side_type", "celltype", "theta", "delta", "vof", "inv_vof", "xtype", "ytype",
          "ztype", "vof_x", "vof_y", "vof_z", "inv_mx", "inv_my", "inv_mz", "dib_en", "dib_ws", "dib_nb", "dib_st",
          "dib_max", "inv_dib_ne", "inv_dib_tn"]


def _bodies(g):
    from lsstag_b200 import mesh as MS
    sph = [tuple(s) for s in g["spheres"].reshape(-1, 4)]
    ell = [(e[0:3], e[3:6], e[6:15].reshape(3, 3)) for e in g["ellipsoids"].reshape(-1, 15)]
    return MS.bodies_array(sph, ell)


def _differences(s, g, fields):
    bad = {}
    for k in fields:
        mine = s.mesh_get(k)
        ref = np.asarray(g[k]).reshape(-1)
        if mine.tobytes() != ref.astype(mine.dtype).tobytes():
            bad[k] = int(np.count_nonzero(mine != ref))
    return bad


@pytest.mark.parametrize("path", CASES, ids=[os.path.basename(p)[5:-4] for p in CASES])
def test_mesh_build_from_bodies_is_bitwise(path):
    from lsstag_b200 import solver as S
    g = dict(np.load(path))
    s = S.MGFGMRES()
    ms = s.build_mesh(g["dims"], g["h"], g["ls_block"], bodies=_bodies(g))
    assert ms > 0
    assert _differences(s, g, FIELDS) == {}
    assert s.ctx.lib.lsg_mesh_osc_sweeps(s.ctx.h) >= 1
    s.close()


@pytest.mark.parametrize("path", CASES[:3], ids=[os.path.basename(p)[5:-4] for p in CASES[:3]])
def test_mesh_build_from_level_set_is_bitwise(path):
    """The same build from the task's own level set (phi given)."""
    from lsstag_b200 import solver as S
    g = dict(np.load(path))
    s = S.MGFGMRES()
    s.build_mesh(g["dims"], g["h"], g["ls_block"], phi=g["phi_ls"])
    assert _differences(s, g, FIELDS) == {}
    s.close()


def test_operator_from_device_mesh_matches_reference_csr():
    """sphere16: the pressure operator assembled from the device mesh equals
    the reference's CSR bit for bit (tests/golden/sphere16.npz holds the
    reference's assembly of the same case), and the MG-FGMRES solve on it
    matches the reference's solve."""
    from lsstag_b200 import solver as S
    from conftest import load_golden, golden_csr
    g = dict(np.load(os.path.join(GOLDEN, "mesh_sphere16.npz")))
    ref = load_golden("sphere16")
    dims = tuple(int(v) for v in ref["dims"])
    s = S.MGFGMRES()
    s.build_mesh(g["dims"], g["h"], g["ls_block"], bodies=_bodies(g))
    s.set_from_mesh(ref["pins"], task=S.Task(eps=float(ref["eps"][0])))
    P = s.planes()
    import ref_runner as rr
    Pref = rr.csr_to_planes(ref["A_rowptr"], ref["A_col"], ref["A_val"], dims)
    assert P.tobytes() == Pref.tobytes()
    x = np.zeros(ref["b"].size)
    it = s.solve(ref["b"], x)
    assert abs(it - int(ref["fgmres_it"][0])) <= 1
    assert np.linalg.norm(x - ref["fgmres_x"]) <= 1e-10 * np.linalg.norm(ref["fgmres_x"])
    assert golden_csr(ref).shape[0] == x.size
    s.close()


def test_four_spheres_128_operator_from_seed():
    """The 128^3 four-sphere Poisson case (seed 3) built on the GPU from the
    seeded spheres alone: its operator equals the reference's assembly stored
    in cases/spheres4_seed3_128.npz, bit for bit."""
    from lsstag_b200 import cases, synth
    from lsstag_b200 import mesh as MS
    from lsstag_b200 import solver as S
    P, dims, pins, _ = cases.load(128)
    h = (1.0 / 128,) * 3
    sph = synth.four_spheres(3)
    s = S.MGFGMRES()
    ms = s.build_mesh(dims, h, MS.flow_block(dims, h, sph), bodies=MS.bodies_array(sph))
    s.set_from_mesh(pins, setup=False)
    mine = s.planes()
    print(f"128^3 four-sphere mesh build: {ms:.3f} ms on the device")
    assert mine.tobytes() == P.tobytes()
    s.close()


def test_flow_case_from_bodies_matches_reference_case():
    """The 128x64x64 sphere flow set up from the sphere alone
    (cases.flow_case_on_device: mesh built on the GPU) equals the case file
    made from the reference's own mesh build and equation set-up, array by
    array and bit for bit, parameters and initial state included."""
    from lsstag_b200 import cases
    g_ref, dims_ref, par_ref, st_ref = cases.load_flow_case()
    h = 1.0 / 16
    g, dims, par, st = cases.flow_case_on_device((128, 64, 64), (h, h, h),
                                                 spheres=[(2.0, 2.0 + 0.5 * h, 2.0 + 0.5 * h, 0.5)])
    assert dims == tuple(dims_ref)
    bad = [k for k in ("celltype", "xtype", "ytype", "ztype", "side_type", "theta", "alpha", "delta", "inv_vof",
                       "vof_x", "vof_y", "vof_z", "inv_mx", "inv_my", "inv_mz", "dib_en", "dib_ws", "dib_nb",
                       "dib_st", "inv_dib_ne", "inv_dib_tn", "vib", "vibyx", "vibzy", "u_w", "bc", "pins", "cells",
                       "dmax", "dne", "dtn")
           if np.asarray(g[k]).reshape(-1).astype(np.asarray(g_ref[k]).dtype).tobytes()
           != np.asarray(g_ref[k]).reshape(-1).tobytes()]
    assert bad == []
    assert float(g["fcoef"]) == float(g_ref["fcoef"])
    for k in ("nu", "coef", "coef2", "coef_integr", "dt", "eps", "vbase", "max_it", "restart_mom", "restart_p"):
        assert par[k] == par_ref[k], k
    for a, b in zip(st, st_ref):
        assert a.tobytes() == np.asarray(b, dtype=np.float64).tobytes()
