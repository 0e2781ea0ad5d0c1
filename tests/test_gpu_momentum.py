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


@pytest.mark.parametrize("name", ["sphere16", "sphere20x12x10"])
def test_momentum_step_matches_reference(name):
    """One momentum step on the GPU: the right-hand side (lsg_momentum_rhs,
    gradient from the geometry, convective product in CSR order) equals the
    reference's bit for bit; ILU-FGMRES(13) on it gives the reference's
    iteration count (+-1) and solution (relative L2 <= 1e-10)."""
    from lsstag_b200 import solver as S
    g = load_golden(name)
    dims = tuple(int(v) for v in g["dims"])
    geo = S.MGFGMRES()
    geom = {k: g[k] for k in ("celltype", "theta", "delta", "inv_mx", "inv_my", "inv_mz")}
    geo.set_geometry(geom, dims, g["pins"], setup=False)
    geo.set_staggered_types(g["xtype"], g["ytype"], g["ztype"])
    for k, d in enumerate("xyz"):
        # the history term left by set(): C(u0) u0 + flux2 in the reference's
        # summation order (the aux output of the same kernel on the first state)
        C0 = (g[f"C{d}_rowptr"], g[f"C{d}_col"], g[f"C{d}_val"])
        _, prev = geo.momentum_rhs(k, C0, g["flux2_0" + d], g["u0" + d], g["u0" + d], g["mstep_vof_" + d],
                                   g["mstep_hflux_" + d], g["mstep_p"], np.zeros_like(g["u0" + d]),
                                   float(g["mstep_coef2"][0]))
        n0 = C0[0].size - 1
        ref_prev = sp.csr_matrix((C0[2], C0[1], C0[0]), shape=(n0, n0)) @ g["u0" + d] + g["flux2_0" + d]
        assert np.linalg.norm(prev - ref_prev) <= 1e-13 * np.linalg.norm(ref_prev)
        right, aux = geo.momentum_rhs(k, (g[f"C1{d}_rowptr"], g[f"C1{d}_col"], g[f"C1{d}_val"]),
                                      g["flux2_1" + d], g["mstep_u_" + d], g["mstep_uprev_" + d],
                                      g["mstep_vof_" + d], g["mstep_hflux_" + d], g["mstep_p"], prev,
                                      float(g["mstep_coef2"][0]))
        assert np.array_equal(right.view(np.int64), g["mstep_rhs_" + d].view(np.int64)), d
        rp, col, val, sdims = _csr(g, "K" + d)
        s = S.ILUFGMRES()
        s.set((rp, col, val, sdims), task=S.Task(eps=1e-10, MAX_ITER=200, FGMRES_RESTART_NUM=int(g["mom_restart"][0])))
        x = np.zeros(rp.size - 1)
        it = s.solve(right, x)
        assert abs(it - int(g["mstep_it_" + d][0])) <= 1, d
        ref = g["mstep_sol_" + d]
        assert np.linalg.norm(x - ref) <= 1e-10 * np.linalg.norm(ref), d
        s.close()
    geo.close()


@pytest.mark.parametrize("name", ["sphere16", "sphere20x12x10"])
def test_convective_apply_bitwise(name):
    """lsg_convective_apply (the convective operator built from the velocity
    on the GPU, matrix-free) equals flux2 + C v of the reference's assembled
    operator bit for bit, and equals the convective product inside
    lsg_momentum_rhs."""
    import lsg_oracle as lo
    from lsstag_b200 import solver as S
    g = load_golden(name)
    dims = tuple(int(v) for v in g["dims"])
    geo = S.MGFGMRES()
    geom = {k: g[k] for k in ("celltype", "theta", "delta", "inv_mx", "inv_my", "inv_mz")}
    geo.set_geometry(geom, dims, g["pins"], setup=False)
    geo.set_staggered_types(g["xtype"], g["ytype"], g["ztype"])
    U = [g["mstep_u_x"], g["mstep_u_y"], g["mstep_u_z"]]
    rng = np.random.default_rng(22)
    for k, d in enumerate("xyz"):
        C = (g[f"C1{d}_rowptr"], g[f"C1{d}_col"], g[f"C1{d}_val"])
        v = rng.standard_normal(C[0].size - 1)
        out = geo.convective_apply(k, U, v, init=g["flux2_1" + d])
        ref = lo._mv(C, v, init=g["flux2_1" + d])
        assert np.array_equal(out.view(np.int64), ref.view(np.int64)), d
        # the history term of the momentum right-hand side from the same product
        aux_mf = geo.convective_apply(k, U, U[k], init=g["flux2_1" + d])
        _, aux = geo.momentum_rhs(k, C, g["flux2_1" + d], U[k], g["mstep_uprev_" + d], g["mstep_vof_" + d],
                                  g["mstep_hflux_" + d], g["mstep_p"], np.zeros_like(U[k]),
                                  float(g["mstep_coef2"][0]))
        assert np.array_equal(aux_mf.view(np.int64), aux.view(np.int64)), d
    geo.close()
