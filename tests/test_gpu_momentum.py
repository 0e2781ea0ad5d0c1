"""The momentum equations' operators on the GPU: the Helmholtz and convective
operators the reference assembles on the staggered x-, y-, z-grids, applied
through the C ABI, and the momentum solve (ILU(0)-FGMRES(13), the reference's
ILUFGMRES) against the reference's own solutions."""
import numpy as np
import pytest
import scipy.sparse as sp

from conftest import GOLDEN_CASES, load_golden

pytestmark = pytest.mark.gpu


def _csr(g, name):
    rp, col, val = g[name + "_rowptr"], g[name + "_col"], g[name + "_val"]
    dims = tuple(int(v) for v in g[name + "_dims"][:3])
    return rp, col, val, dims


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_momentum_operator_apply(name):
    """y = K u and y = C u on the staggered grids, against the CSR product
    (relative 1e-14)."""
    from lsstag_b200 import solver as S
    g = load_golden(name)
    rng = np.random.default_rng(2)
    for d in "xyz":
        for m in ("K", "C"):
            rp, col, val, dims = _csr(g, m + d)
            n = rp.size - 1
            A = sp.csr_matrix((val, col, rp), shape=(n, n))
            u = rng.standard_normal(n)
            s = S.ILUFGMRES()
            s.set((rp, col, val, dims), setup=False)
            y = s.apply(u)
            ref = A @ u
            assert np.linalg.norm(y - ref) <= 1e-14 * np.linalg.norm(ref), (m, d)
            s.close()


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_momentum_solve_matches_reference(name):
    """ILU-FGMRES(13) on each Helmholtz system: the reference's iteration
    count (+-1) and solution (relative L2 <= 1e-10)."""
    from lsstag_b200 import solver as S
    g = load_golden(name)
    for d in "xyz":
        rp, col, val, dims = _csr(g, "K" + d)
        s = S.ILUFGMRES()
        s.set((rp, col, val, dims), task=S.Task(eps=float(g[f"mom_eps_{d}"][0]), MAX_ITER=200,
                                                FGMRES_RESTART_NUM=int(g["mom_restart"][0])))
        x = np.zeros(rp.size - 1)
        it = s.solve(g[f"mom_rhs_{d}"], x)
        assert abs(it - int(g[f"mom_it_{d}"][0])) <= 1, d
        ref = g[f"mom_x_{d}"]
        assert np.linalg.norm(x - ref) <= 1e-10 * np.linalg.norm(ref), d
        s.close()
