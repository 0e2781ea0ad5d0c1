"""Operator set of the flow time step built from the CPU restatement (the
oracle), for checking lsstag_b200.flow_adjoint's reverse sweep without a GPU:
the same methods as flow_adjoint.GpuFlowOps, with the oracle's
laplace_flux / convective_flux / convective_apply / helmholtz_flux /
projection_rhs / projection_correct / loads_forces and their transposes
(convective_adjoint, loads_adjoint, scipy transposes of the divergence and
gradient matrices), and exact sparse LU solves in place of the Krylov solves
(the pressure solve on the rows that are not pinned to zero)."""
import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spl

import lsg_oracle as lo

from lsstag_b200 import flow_adjoint as FA


def planes_csr(P, dims):
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


def _csr(t, shape=None):
    rp, col, val = t
    nrow = rp.size - 1
    return sp.csr_matrix((val, col, rp), shape=shape or (nrow, int(col.max()) + 1 if col.size else 0))


def load_adjoint_case():
    """(geom, dims, par) of the 16^3 sphere flow with the loads inputs of the
    same geometry."""
    from conftest import load_golden
    g = load_golden("flow16_steps")
    ld = load_golden("loads_sphere16")
    for k in ("celltype", "theta", "delta", "inv_vof"):
        assert np.array_equal(g[k], ld[k])
    geom = dict(g)
    for k in ("cells", "dmax", "dne", "dtn", "nodes", "center"):
        geom[k] = ld[k]
    nu, coef, coef2, integr, dt, eps, vbase, maxit = (float(v) for v in g["nu_coef_coef2_integr_dt_eps_vbase_maxit"])
    rm, rp = (int(v) for v in g["restart_mom_p"])
    par = dict(nu=nu, coef=coef, coef2=coef2, coef_integr=integr, dt=dt, eps=eps, vbase=vbase, max_it=maxit,
               restart_mom=rm, restart_p=rp, fcoef=float(ld["nu_fcoef_dt"][1]))
    dims = tuple(int(v) for v in g["dims"])
    return geom, dims, par


class OracleFlowOps:
    def __init__(self, geom, dims, par):
        self.g, self.par = geom, par
        N, M, K = self.dims = tuple(dims)
        self.nu = float(par["nu"])
        self.bc = np.asarray(geom["bc"], dtype=np.float64)
        g = geom
        self.stypes = [np.asarray(g[c + "type"]) for c in "xyz"]
        self.vof = [np.asarray(g["vof_" + c], dtype=np.float64) for c in "xyz"]
        self.inv = (g["inv_mx"], g["inv_my"], g["inv_mz"])
        self.D = lo.divergence_from_geometry(N, M, K, g["celltype"], g["theta"], g["delta"])
        self.G = lo.gradient_from_geometry(N, M, K, g["xtype"], g["ytype"], g["ztype"], g["theta"], g["delta"])
        n = N * M * K
        gd = [FA.grid_dims(d, self.dims) for d in range(3)]
        self.Ds = [_csr(t, (n, int(np.prod(gd[d])))) for d, t in enumerate(self.D)]
        self.Gs = [_csr(t, (int(np.prod(gd[d])), n)) for d, t in enumerate(self.G)]
        A = planes_csr(lo.laplace_from_geometry(N, M, K, g["celltype"], g["theta"], g["delta"], g["inv_mx"],
                                                g["inv_my"], g["inv_mz"], g["pins"]), self.dims).tocsr()
        # the pinned rows are empty; solid cells hold only a 1e-16 diagonal and
        # a zero right-hand side: the live block is solved exactly, the rest is 0
        self.live = (A.diagonal() != 0) & (np.asarray(g["celltype"]) != lo.SOLID_CELL)
        Ass = A[self.live][:, self.live].tocsc()
        self.A_lu, self.AT_lu = spl.splu(Ass), spl.splu(Ass.T.tocsc())
        self.H_lu = []
        for d, c in enumerate("xyz"):
            rp, col, val = lo.helmholtz_from_geometry(d, N, M, K, g[c + "type"], g["theta"], g["alpha"], g["delta"],
                                                      g["inv_vof"], g["vof_" + c], g["dib_en"], g["dib_ws"],
                                                      g["dib_nb"], g["dib_st"], g["inv_dib_ne"], g["inv_dib_tn"],
                                                      self.nu, par["coef_integr"], True)
            H = sp.csr_matrix((val, col, rp), shape=(rp.size - 1, rp.size - 1))
            # solid rows hold only a 1e-16 diagonal and a zero right-hand side:
            # the fluid block is solved exactly, the solid rows give 0
            fl = self.stypes[d] != 0
            Hff = H[fl][:, fl].tocsc()
            self.H_lu.append((fl, spl.splu(Hff), spl.splu(Hff.T.tocsc()), H.diagonal()))
        self.set_inflow(g["u_w"])

    def set_inflow(self, u_w):
        N, M, K = self.dims
        self.u_w = np.asarray(u_w, dtype=np.float64)
        self.hflux = [lo.helmholtz_flux(d, N, M, K, self.stypes[d], self.g["delta"], self.u_w, self.bc, self.nu)
                      for d in range(3)]

    def laplace_flux(self, ux):
        N, M, K = self.dims
        g, bc = self.g, self.bc
        return lo.laplace_flux(N, M, K, g["celltype"], g["side_type"], g["theta"], g["delta"], g["vib"], self.u_w,
                               bc[1], bc[8], bc[9], bc[16], bc[17], ux)

    def conv_term(self, d, u):
        N, M, K = self.dims
        g = self.g
        f2 = lo.convective_flux(d, N, M, K, g["theta"], g["delta"], *u, self.u_w, self.bc)
        return lo.convective_apply(d, N, M, K, self.stypes[d], g["theta"], g["delta"], u, u[d], init=f2)

    def momentum_rhs(self, d, c, ud, uprevd, p, prev_aux_d):
        right = (-2.0 * ud + 0.5 * uprevd) * self.vof[d] * self.par["coef2"]
        right = right - ((lo._mv(self.G[d], p) + self.hflux[d]) + prev_aux_d)
        return right + c * 2.0

    def helm_solve(self, d, right, x0):
        fl, lu, _, diag = self.H_lu[d]
        right = np.asarray(right, dtype=np.float64)
        x = right / diag
        x[fl] = lu.solve(right[fl])
        return x

    def projection_rhs(self, s, L):
        return lo.projection_rhs(self.D, s[0], s[1], s[2], L, self.g["pins"])

    def pressure_solve(self, b):
        x = np.zeros_like(b)
        x[self.live] = self.A_lu.solve(b[self.live])
        return x

    def projection_correct(self, phi, s, p, outflow):
        N, M, K = self.dims
        u, v, w, pn = lo.projection_correct(self.G, self.inv, phi, s[0], s[1], s[2], np.array(p, copy=True),
                                            self.par["coef"], N, M, K, self.par["vbase"], outflow)
        return [u, v, w], pn

    def _loads_args(self):
        g = self.g
        N, M, K = self.dims
        return (N, M, K, g["cells"], g["celltype"], g["theta"], g["delta"], g["inv_vof"], g["dmax"], g["dne"],
                g["dtn"])

    def drag(self, u, p):
        g = self.g
        fx, _, _ = lo.loads_forces(*self._loads_args(), g["vib"], g["vibyx"], g["vibzy"], u[0], u[1], u[2], p,
                                   self.nu)
        return fx.sum() * self.par["fcoef"]

    def drag_gradient(self):
        gx, gy, gz, gp = lo.loads_adjoint(*self._loads_args(), (self.par["fcoef"], 0.0, 0.0), self.nu)
        return [gx, gy, gz], gp

    def projection_adjoint(self, qbar, pbar):
        phib = sum(self.Gs[d].T @ (np.asarray(self.inv[d]) * qbar[d]) for d in range(3)) + self.par["coef"] * pbar
        lam = np.zeros_like(phib)
        lam[self.live] = self.AT_lu.solve(phib[self.live])
        for p in self.g["pins"]:
            lam[int(p)] = 0.0
        return [qbar[d] + self.Ds[d].T @ lam for d in range(3)], lam

    def helm_solve_T(self, d, g):
        fl, _, luT, _ = self.H_lu[d]
        x = np.zeros(np.asarray(g).size)
        x[fl] = luT.solve(np.asarray(g, dtype=np.float64)[fl])
        return x

    def gradient_T(self, r):
        return sum(self.Gs[d].T @ r[d] for d in range(3))

    def conv_adjoint(self, d, u, cbar):
        N, M, K = self.dims
        Ub, vb = lo.convective_adjoint(d, N, M, K, self.stypes[d], self.g["theta"], self.g["delta"], u, u[d], cbar)
        Ub[d] = Ub[d] + vb
        return Ub

    def close(self):
        pass
