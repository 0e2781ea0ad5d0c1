"""GPU assembly of the cut-cell Laplace operator from the geometry
(lsg_set_matrix_geometry) against the reference's own CSR, bit for bit."""
import numpy as np
import pytest

import ref_runner as rr
from conftest import GOLDEN_CASES, load_golden

pytestmark = pytest.mark.gpu


def _geom(g):
    return {k: g[k] for k in ("celltype", "theta", "delta", "inv_mx", "inv_my", "inv_mz")}


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_assembly_bitwise(name):
    from lsstag_b200 import solver as S
    g = load_golden(name)
    dims = tuple(int(v) for v in g["dims"])
    s = S.MGFGMRES()
    s.set_geometry(_geom(g), dims, g["pins"], task=S.Task(eps=float(g["eps"][0])), setup=False)
    P = s.planes()
    ref = rr.csr_to_planes(g["A_rowptr"], g["A_col"], g["A_val"], dims)
    assert np.array_equal(P.view(np.int64), ref.view(np.int64))
    s.close()


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_assembled_solve_matches_reference(name):
    """MG-FGMRES on the GPU-assembled operator: the reference's iteration
    count (+-1) and solution (relative L2 <= 1e-10)."""
    from lsstag_b200 import solver as S
    g = load_golden(name)
    dims = tuple(int(v) for v in g["dims"])
    s = S.MGFGMRES()
    s.set_geometry(_geom(g), dims, g["pins"], task=S.Task(eps=float(g["eps"][0]), MAX_ITER=200,
                                                          FGMRES_RESTART_NUM=30))
    x = np.zeros_like(g["b"])
    it = s.solve(g["b"], x)
    assert abs(it - int(g["fgmres_it"][0])) <= 1
    assert np.linalg.norm(x - g["fgmres_x"]) <= 1e-10 * np.linalg.norm(g["fgmres_x"])
    s.close()


def test_assembly_rejects_bad_arguments():
    from lsstag_b200 import _lib as L
    ctx = L.Context(0)
    rc = ctx.lib.lsg_set_matrix_geometry(ctx.h, 1, 4, 4, None, None, None, None, None, None, 0, 0)
    assert rc == L.LSG_ERR_ARG
    ctx.close()
