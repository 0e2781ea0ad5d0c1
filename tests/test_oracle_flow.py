"""Whole time steps of the flow past the 16^3 sphere composed from the CPU
restatement (laplace_flux, convective_flux, convective_apply, the momentum
right-hand side, helmholtz_from_geometry / helmholtz_flux with ILU(0)-FGMRES,
the projection right-hand side, MG-FGMRES and projection_correct) in the order
of TimeSteppingMethodInterface::step (time_stepping_method_interface.h:172-214)
against the reference's own three steps: iterations within 1, states within
1e-9 relative L2 (both sides solve to an absolute residual of 1e-11)."""
import numpy as np
import scipy.sparse as sp

from conftest import load_golden

import lsg_oracle as lo


def _planes_csr(P, dims):
    N, M, K = dims
    n = N * M * K
    NM = N * M
    i = np.arange(n)
    x, y, z = i % N, (i // N) % M, i // NM
    offs = [-NM, -N, -1, 0, 1, N, NM]
    ok = [z > 0, y > 0, x > 0, np.ones(n, bool), x < N - 1, y < M - 1, z < K - 1]
    rows, cols, vals = [], [], []
    for s in range(7):
        rows.append(i[ok[s]])
        cols.append(i[ok[s]] + offs[s])
        vals.append(P[s][ok[s]])
    return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def test_oracle_flow_steps_match_reference():
    g = load_golden("flow16_steps")
    N, M, K = dims = tuple(int(v) for v in g["dims"])
    nu, coef, coef2, integr, dt, eps, vbase, maxit = (float(v) for v in g["nu_coef_coef2_integr_dt_eps_vbase_maxit"])
    rmom, rp_ = (int(v) for v in g["restart_mom_p"])
    bc = g["bc"]
    D = lo.divergence_from_geometry(N, M, K, g["celltype"], g["theta"], g["delta"])
    G = lo.gradient_from_geometry(N, M, K, g["xtype"], g["ytype"], g["ztype"], g["theta"], g["delta"])
    A = _planes_csr(lo.laplace_from_geometry(N, M, K, g["celltype"], g["theta"], g["delta"], g["inv_mx"], g["inv_my"],
                                             g["inv_mz"], g["pins"]), dims)
    mg = lo.MultiGrid(A, dims)
    Ks, LUs, hflux = [], [], []
    for d, c in enumerate("xyz"):
        rp, col, val = lo.helmholtz_from_geometry(d, N, M, K, g[c + "type"], g["theta"], g["alpha"], g["delta"],
                                                  g["inv_vof"], g["vof_" + c], g["dib_en"], g["dib_ws"], g["dib_nb"],
                                                  g["dib_st"], g["inv_dib_ne"], g["inv_dib_tn"], nu, integr, True)
        Kd = sp.csr_matrix((val, col, rp), shape=(rp.size - 1, rp.size - 1))
        Ks.append(Kd)
        LUs.append(lo.ilu0(Kd))
        hflux.append(lo.helmholtz_flux(d, N, M, K, g[c + "type"], g["delta"], g["u_w"], bc, nu))
    stypes = [g["xtype"], g["ytype"], g["ztype"]]
    u = [g["u_0"].copy(), g["v_0"].copy(), g["w_0"].copy()]
    p = g["p_0"].copy()

    def conv(d):
        f2 = lo.convective_flux(d, N, M, K, g["theta"], g["delta"], *u, g["u_w"], bc)
        return lo.convective_apply(d, N, M, K, stypes[d], g["theta"], g["delta"], u, u[d], init=f2)

    uprev = [a.copy() for a in u]           # HelmholtzDiscreteEquation::set: previous = current
    prev_aux = [conv(d) for d in range(3)]
    for s in (1, 2, 3):
        flux_lap = lo.laplace_flux(N, M, K, g["celltype"], g["side_type"], g["theta"], g["delta"], g["vib"],
                                   g["u_w"], bc[1], bc[8], bc[9], bc[16], bc[17], u[0])
        us, its = [], []
        for d, c in enumerate("xyz"):
            aux = conv(d)
            right = (-2.0 * u[d] + 0.5 * uprev[d]) * g["vof_" + c] * coef2
            right = right - ((lo._mv(G[d], p) + hflux[d]) + prev_aux[d])
            right = right + aux * 2.0
            prev_aux[d] = aux
            x, it, _ = lo.fgmres(Ks[d], right, u[d].copy(), lambda v, LU=LUs[d]: lo.ilu_solve(LU, v), eps, rmom,
                                 int(maxit))
            us.append(x)
            its.append(it)
        b = lo.projection_rhs(D, us[0], us[1], us[2], flux_lap, g["pins"])
        phi, itp, _ = lo.fgmres(A, b, np.zeros_like(p), mg.apply, eps, rp_, int(maxit))
        its.append(itp)
        for a, r in zip(its, g[f"its_{s}"]):
            assert abs(int(a) - int(r)) <= 1, (s, its, g[f"its_{s}"])
        uprev = [a.copy() for a in u]
        un, vn, wn, p = lo.projection_correct(G, (g["inv_mx"], g["inv_my"], g["inv_mz"]), phi, us[0], us[1], us[2],
                                              p, coef, N, M, K, vbase)
        u = [un, vn, wn]
        for name, mine in zip("uvw", u):
            assert _rel(mine, g[f"{name}_{s}"]) <= 1e-9, (s, name, _rel(mine, g[f"{name}_{s}"]))
        assert _rel(p, g[f"p_{s}"]) <= 1e-9, (s, "p")
