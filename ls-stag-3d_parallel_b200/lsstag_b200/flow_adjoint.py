"""Discrete adjoint of the fixed-body flow's time steps: the gradient of the
time-averaged drag coefficient with respect to an inflow profile and a
momentum forcing field, through S time steps recomputed from checkpoints.
The reference has no adjoint; the forward map is its time step
(TimeSteppingMethodInterface::step, time_stepping_method_interface.h:172-214)
as FlowStepper runs it.

Objective and parameters
  J = (1/S) sum_{n=1..S} C_d(u^n, p^n),  C_d = fcoef F_aer_x of
      LoadsCalculator::calculate (loads_calculator.h:1366-1377), unfiltered;
  theta (8): the inflow profile u_w = u_w0 + sum_k theta_k phi_k, u_w the
      per-(y, z) x-inflow array pU_W (base_task_description.h:313-315) that
      the pressure source term, the x-momentum source term and the z
      convective source term read; phi_k = sin(a pi y') sin(b pi z') at the
      inflow face's cell centres y' = (j + 1/2)/M, z' = (k + 1/2)/K for
      (a, b) in INFLOW_MODES;
  f = (f_x, f_y, f_z): a forcing field on the three staggered grids, added
      to every momentum right-hand side as VOF_d f_d on fluid faces (zero on
      solid faces, where the velocity stays 0).

One forward step n maps (u^n, u^{n-1}, p^n, a^{n-1}) -- a the Adams-Bashforth
history flux2 + C(u) u of each momentum equation -- to the next state:
  L = laplace_flux(u_w, u^n_x);  c_d = flux2_d(u^n, u_w) + C_d(u^n) u^n_d;
  r_d = (-2 u^n_d + 1/2 u^{n-1}_d) VOF_d / dt - (G_d p^n + h_d(u_w) + a^{n-1}_d) + 2 c_d + VOF_d f_d;
  s_d = H_d^{-1} r_d;  phi = A^{-1} (D s + L, pins 0);
  u^{n+1} = clamp(G phi / VOF + s);  p^{n+1} = p^n + 1.5/dt phi;  a^n = c.
The reverse step applies the transposes in the opposite order: the clamp
mask, the projection adjoint (G^T, A^T solve, D^T), the transposed momentum
solves H_d^T, G^T for the pressure term, the transposed convective Jacobian
and the transposes of the three source terms.  Checkpoints of the state are
kept every `every` steps; each segment is recomputed once in the reverse
sweep, recording u^n and the clamp masks.

The operators come from an operator set (GpuFlowOps: every operator and
every transposed operator through the C ABI on the GPU).  The boundary
source terms' transposes (O(M K + N M) entries) and the clamp mask are
evaluated here on the host from the geometry.
"""
from __future__ import annotations

import numpy as np

from . import solver as S

INFLOW_MODES = ((1, 1), (1, 2), (2, 1), (2, 2), (1, 3), (3, 1), (2, 3), (3, 2))


def inflow_basis(M: int, K: int) -> np.ndarray:
    """(8, M*K): the inflow modes phi_k at index y + z*M (the layout of pU_W)."""
    y = (np.arange(M) + 0.5) / M
    z = (np.arange(K) + 0.5) / K
    B = np.empty((len(INFLOW_MODES), M * K))
    for k, (a, b) in enumerate(INFLOW_MODES):
        B[k] = (np.sin(b * np.pi * z)[:, None] * np.sin(a * np.pi * y)[None, :]).ravel()
    return B


def grid_dims(d: int, dims):
    N, M, K = dims
    return (N - (d == 0), M - (d == 1), K - (d == 2))


def outflow_clamp_mask(dims, qx, qy, qz):
    """Entries that the outflow clamps of SetSolutions::correction
    (corrOutFlow / corrOutFlowTB, Base/set_solutions.h:87-118, :297-304)
    overwrite with constants, from the velocities before the clamps: per
    interior (y, z) row of the east outflow, if the last x-face value is
    negative it becomes V_BASE and the row's last y- and z-faces 0 (likewise
    the face before it); a bottom z-face with positive or a top z-face with
    negative velocity becomes 0.  Returns boolean masks on the three grids."""
    N, M, K = dims
    NM = N * M
    mx, my, mz = (np.zeros(np.asarray(a).size, dtype=bool) for a in (qx, qy, qz))
    zz, yy = np.meshgrid(np.arange(1, K - 1), np.arange(1, M - 1), indexing="ij")
    zz, yy = zz.ravel(), yy.ravel()
    num = (yy + 1) * N - 1 + zz * NM
    num2 = num - yy - 1 - zz * M
    num3 = num - zz * N
    for sh in (0, 1):
        hit = qx[num2 - sh] < 0.0
        mx[(num2 - sh)[hit]] = True
        my[(num3 - sh)[hit]] = True
        mz[(num - sh)[hit]] = True
    yy, xx = np.meshgrid(np.arange(1, M), np.arange(1, N), indexing="ij")
    nb = (xx + yy * N).ravel()
    nt = nb + (K - 2) * NM
    mz[nb[qz[nb] > 0.0]] = True
    mz[nt[qz[nt] < 0.0]] = True
    return mx, my, mz


class SourceTermTransposes:
    """Transposes of the boundary source terms that depend on the inflow
    profile or the velocity, as the forward computes them:
      laplace flux (LaplaceDiscreteOperator calcFlux / setBaseFlux,
        laplace_discrete_operator.h:47-83, :687-808): -u_w dy dz at x = 0,
        u_x(last x-face) dy dz at x = N-1;
      x-momentum flux (inFlowFluxHelmX, helmholtz_discrete_operator_x.h:50-96):
        u_w nu dz dy / dx at x = 0;
      z convective flux (ConvectiveDiscreteOperatorZ::baseFlux,
        convective_discrete_operator_z.h:748-757): the inflow term
        -(u_w dz + u_w' dz') W_W dy / 4, the outflow term
        u_z (u_x dz + u_x' dz') dy / 4 and the bottom/top terms
        -/+ dx dy theta_z w^2 / 2.
    The other terms are constants of the boundary velocities."""

    def __init__(self, dims, theta, delta, bc, nu: float):
        N, M, K = self.dims = tuple(int(v) for v in dims)
        NM = N * M
        de = np.asarray(delta, dtype=np.float64).reshape(-1, 3)
        th = np.asarray(theta, dtype=np.float64).reshape(-1, 3)
        zz, yy = np.meshgrid(np.arange(K), np.arange(M), indexing="ij")
        zz, yy = zz.ravel(), yy.ravel()
        # laplace flux: inflow rows and outflow rows
        self.lap_in = N * yy + NM * zz
        self.lap_in_w = yy + zz * M
        self.lap_in_c = -(de[self.lap_in, 1] * de[self.lap_in, 2])
        self.lap_out = (yy + 1) * N - 1 + zz * NM
        self.lap_out_u = self.lap_out - 1 - yy - zz * M
        self.lap_out_c = de[self.lap_out, 1] * de[self.lap_out, 2]
        # x-momentum inflow rows
        P = N * yy + NM * zz
        self.hx_row = (N - 1) * M * zz + (N - 1) * yy
        self.hx_w = yy + zz * M
        self.hx_c = nu * de[P, 2] * de[P, 1] / de[P, 0]
        # z convective flux (layers z < K-1)
        zz, yy = np.meshgrid(np.arange(K - 1), np.arange(M), indexing="ij")
        zz, yy = zz.ravel(), yy.ravel()
        numF = N * yy + NM * zz
        numW = yy + zz * M
        dz, dy, dzz = de[numF, 2], de[numF, 1], de[numF + NM, 2]
        W_W = float(np.asarray(bc)[12])
        self.cz_in, self.cz_in_w = numF, numW
        self.cz_in_c0, self.cz_in_c1 = -0.25 * dz * W_W * dy, -0.25 * dzz * W_W * dy
        self.cz_last = numF + N - 1
        self.cz_u0 = self.cz_last - numW - 1
        self.cz_u1 = self.cz_u0 + (N - 1) * M
        self.cz_dz, self.cz_dzz, self.cz_dy = dz, dzz, dy
        yy, xx = np.meshgrid(np.arange(M), np.arange(N), indexing="ij")
        nb = (xx + yy * N).ravel()
        nt = nb + (K - 2) * NM
        self.cz_nb, self.cz_nt = nb, nt
        self.cz_cb = -(de[nb, 0] * de[nb, 1] * th[nb, 2])
        self.cz_ct = de[nt, 0] * de[nt, 1] * th[nt, 2]

    def laplace_flux_T(self, Lbar):
        """(u_x cotangent, u_w cotangent) of <Lbar, laplace_flux(u_w, u_x)>."""
        N, M, K = self.dims
        uxb = np.zeros((N - 1) * M * K)
        np.add.at(uxb, self.lap_out_u, Lbar[self.lap_out] * self.lap_out_c)
        uwb = np.zeros(M * K)
        np.add.at(uwb, self.lap_in_w, Lbar[self.lap_in] * self.lap_in_c)
        return uxb, uwb

    def helmholtz_flux_T(self, hbar_x):
        """u_w cotangent of <hbar_x, h_x(u_w)> (the y and z terms hold no u_w)."""
        N, M, K = self.dims
        uwb = np.zeros(M * K)
        np.add.at(uwb, self.hx_w, hbar_x[self.hx_row] * self.hx_c)
        return uwb

    def convective_flux_T(self, cbar_z, ux, uz):
        """(u_x, u_z, u_w) cotangents of <cbar_z, flux2_z(u, u_w)> at the
        velocities (ux, uz) the forward read."""
        N, M, K = self.dims
        uxb = np.zeros((N - 1) * M * K)
        uzb = np.zeros(N * M * (K - 1))
        uwb = np.zeros(M * K)
        cin = cbar_z[self.cz_in]
        np.add.at(uwb, self.cz_in_w, cin * self.cz_in_c0)
        np.add.at(uwb, self.cz_in_w + M, cin * self.cz_in_c1)
        cl = cbar_z[self.cz_last]
        np.add.at(uzb, self.cz_last,
                  cl * 0.25 * (ux[self.cz_u0] * self.cz_dz + ux[self.cz_u1] * self.cz_dzz) * self.cz_dy)
        w = cl * 0.25 * uz[self.cz_last] * self.cz_dy
        np.add.at(uxb, self.cz_u0, w * self.cz_dz)
        np.add.at(uxb, self.cz_u1, w * self.cz_dzz)
        np.add.at(uzb, self.cz_nb, cbar_z[self.cz_nb] * self.cz_cb * uz[self.cz_nb])
        np.add.at(uzb, self.cz_nt, cbar_z[self.cz_nt] * self.cz_ct * uz[self.cz_nt])
        return uxb, uzb, uwb


def planes_decouple(P: np.ndarray, dims, solid: np.ndarray) -> np.ndarray:
    """The 7 coefficient planes (offsets -NM, -N, -1, 0, 1, N, NM) with every
    coupling to or from a solid row removed (solid rows keep their
    diagonal).  The momentum solution is 0 on solid faces for every right-hand
    side the time step produces, so the forward map is unchanged, while the
    transposed system no longer routes cotangents through the solid rows'
    1e-16 diagonals."""
    N, M, K = dims
    n = N * M * K
    i = np.arange(n)
    offs = (-N * M, -N, -1, 0, 1, N, N * M)
    Q = np.array(P, dtype=np.float64, copy=True)
    for s, o in enumerate(offs):
        if o == 0:
            continue
        j = np.clip(i + o, 0, n - 1)
        Q[s][solid | solid[j]] = 0.0
    return Q


def planes_transpose(P: np.ndarray, dims) -> np.ndarray:
    """Planes of A^T: row i, offset o holds A[i + o, i], the entry of row
    i + o at offset -o (zero toward cells outside the grid)."""
    N, M, K = dims
    n = N * M * K
    i = np.arange(n)
    x, y, z = i % N, (i // N) % M, i // (N * M)
    offs = (-N * M, -N, -1, 0, 1, N, N * M)
    ok = (z > 0, y > 0, x > 0, np.ones(n, bool), x < N - 1, y < M - 1, z < K - 1)
    T = np.zeros_like(P)
    for s, o in enumerate(offs):
        T[s][ok[s]] = P[6 - s][i[ok[s]] + o]
    return T


class GpuFlowOps:
    """Every forward and transposed operator of the time step on the GPU
    through the C ABI: the pressure context (MG-FGMRES; projection, gradient
    transpose, convective operator and its transposed Jacobian), one
    ILU(0)-FGMRES context per momentum equation and one per transposed
    momentum operator, and the loads context for the drag and its gradient.

    geom: FlowStepper's mesh arrays plus the loads inputs cells, dmax (delta_ib_max),
    dne (inv_delta_ib_ne), dtn (inv_delta_ib_tn) and, optionally, nodes and
    center (they enter the moments only, not the drag); par: FlowStepper's
    parameters plus fcoef and dt."""

    def __init__(self, geom: dict, dims, par: dict, device: int = 0):
        from .loads import LoadsCalculator
        self.g, self.par = geom, par
        self.dims = tuple(int(v) for v in dims)
        self.bc = np.asarray(geom["bc"], dtype=np.float64)
        self.bc_lap = self.bc[[1, 8, 9, 16, 17]].copy()
        self.nu = float(par["nu"])
        ptask = S.Task(eps=par["eps"], MAX_ITER=int(par["max_it"]), FGMRES_RESTART_NUM=int(par["restart_p"]))
        self.pres = S.MGFGMRES(device=device)
        self.pres.set_geometry({k: geom[k] for k in ("celltype", "theta", "delta", "inv_mx", "inv_my", "inv_mz")},
                               self.dims, geom["pins"], task=ptask)
        self.pres.set_staggered_types(geom["xtype"], geom["ytype"], geom["ztype"])
        mtask = S.Task(eps=par["eps"], MAX_ITER=int(par["max_it"]), FGMRES_RESTART_NUM=int(par["restart_mom"]))
        self.stypes = [np.asarray(geom[c + "type"]) for c in "xyz"]
        self.vof = [np.asarray(geom["vof_" + c], dtype=np.float64) for c in "xyz"]
        self.mom, self.momT = [], []
        for d, c in enumerate("xyz"):
            hg = {k: geom[k] for k in ("theta", "alpha", "delta", "inv_vof", "dib_en", "dib_ws", "dib_nb", "dib_st",
                                       "inv_dib_ne", "inv_dib_tn")}
            hg["stype"] = geom[c + "type"]
            hg["vof"] = geom["vof_" + c]
            s = S.ILUFGMRES(device=device)
            s.set_helmholtz(d, hg, self.dims, self.nu, par["coef_integr"], True, task=mtask)
            self.mom.append(s)
            gd = grid_dims(d, self.dims)
            PT = planes_transpose(planes_decouple(s.planes(), gd, self.stypes[d] == 0), gd)
            t = S.ILUFGMRES(device=device)
            t.set_planes(PT, gd, task=S.Task(eps=par["eps"], MAX_ITER=int(par["max_it"]),
                                             FGMRES_RESTART_NUM=int(par["restart_mom"])))
            self.momT.append(t)
        self.loads = LoadsCalculator(device=device)
        n = int(np.prod(self.dims))
        self.loads.set(self.dims, geom["cells"], geom["celltype"], geom["theta"], geom["delta"], geom["inv_vof"],
                       geom["dmax"], geom["dne"], geom["dtn"], geom.get("nodes", np.zeros(3 * n)),
                       geom.get("center", np.zeros(3)), par["fcoef"], par["dt"])
        self.set_inflow(geom["u_w"])

    def set_inflow(self, u_w):
        self.u_w = np.ascontiguousarray(u_w, dtype=np.float64)
        self.hflux = [self.mom[d].helmholtz_flux(d, self.dims, self.g["xyz"[d] + "type"], self.g["delta"], self.u_w,
                                                 self.bc, self.nu) for d in range(3)]

    def laplace_flux(self, ux):
        return self.pres.laplace_flux(self.g["side_type"], self.g["vib"], self.u_w, self.bc_lap, ux)

    def conv_term(self, d, u):
        flux2 = self.mom[d].convective_flux(d, self.dims, self.g["theta"], self.g["delta"], *u, self.u_w, self.bc)
        return self.pres.convective_apply(d, u, u[d], init=flux2)

    def momentum_rhs(self, d, c, ud, uprevd, p, prev_aux_d):
        right, _ = self.pres.momentum_rhs(d, None, c, ud, uprevd, self.vof[d], self.hflux[d], p, prev_aux_d,
                                          self.par["coef2"])
        return right

    def helm_solve(self, d, right, x0):
        x = np.array(x0, dtype=np.float64, copy=True)
        self.mom[d].solve(right, x)
        return x

    def projection_rhs(self, s, L):
        return self.pres.projection_rhs(s[0], s[1], s[2], L)

    def pressure_solve(self, b):
        phi = np.zeros_like(b)
        self.pres.solve(b, phi)
        return phi

    def projection_correct(self, phi, s, p, outflow):
        pn = np.array(p, dtype=np.float64, copy=True)
        u, v, w, pn = self.pres.projection_correct(phi, s[0], s[1], s[2], pn, self.par["coef"], self.par["vbase"],
                                                   outflow)
        return [u, v, w], pn

    def drag(self, u, p):
        g = self.g
        return self.loads.calculate(u[0], u[1], u[2], p, g["vib"], g["vibyx"], g["vibzy"], self.nu).coef[0]

    def drag_gradient(self):
        gx, gy, gz, gp = self.loads.adjoint((float(self.par["fcoef"]), 0.0, 0.0), self.nu)
        return [gx, gy, gz], gp

    def projection_adjoint(self, qbar, pbar):
        ub, vb, wb, fb, _ = self.pres.projection_adjoint(qbar[0], qbar[1], qbar[2], pbar, self.par["coef"])
        return [ub, vb, wb], fb

    def helm_solve_T(self, d, g):
        x = np.zeros_like(g)
        self.momT[d].solve(g, x)
        return x

    def gradient_T(self, r):
        return self.pres.gradient_transpose(r[0], r[1], r[2])

    def conv_adjoint(self, d, u, cbar):
        ub = self.pres.convective_adjoint(d, u, u[d], cbar)
        out = [ub[0], ub[1], ub[2]]
        out[d] = out[d] + ub[3]
        return out

    def close(self):
        for s in self.mom + self.momT:
            s.close()
        self.pres.close()
        self.loads.close()


class FlowAdjoint:
    """J(theta, f) over `steps` time steps from the state (u0, p0) and its
    gradient by the discrete adjoint, checkpoints every `every` steps.

    ops: the operator set (GpuFlowOps).  Its attributes dims, stypes, vof, par
    (coef, coef2), g (theta, delta, bc, u_w) and nu are read here."""

    def __init__(self, ops, steps: int, every: int = 10):
        self.ops = ops
        self.S = int(steps)
        self.every = max(1, int(every))
        N, M, K = self.dims = ops.dims
        self.B = inflow_basis(M, K)
        self.u_w0 = np.asarray(ops.g["u_w"], dtype=np.float64).copy()
        self.fluid = [np.asarray(t) != 0 for t in ops.stypes]
        self.fvof = [np.where(f, v, 0.0) for f, v in zip(self.fluid, ops.vof)]
        self.src = SourceTermTransposes(self.dims, ops.g["theta"], ops.g["delta"], ops.g["bc"], ops.nu)
        self.checkpoints = {}
        self.stats = {}

    # -- forward -------------------------------------------------------------
    def _initial(self, u0, p0):
        u = [np.array(a, dtype=np.float64, copy=True) for a in u0]
        return (u, [a.copy() for a in u], np.array(p0, dtype=np.float64, copy=True),
                [self.ops.conv_term(d, u) for d in range(3)])

    def _step(self, st, forcing, rec=None):
        ops = self.ops
        u, uprev, p, pa = st
        L = ops.laplace_flux(u[0])
        s, c = [], []
        for d in range(3):
            cd = ops.conv_term(d, u)
            right = ops.momentum_rhs(d, cd, u[d], uprev[d], p, pa[d])
            if forcing is not None:
                right = right + self.fvof[d] * forcing[d]
            s.append(ops.helm_solve(d, right, u[d]))
            c.append(cd)
        phi = ops.pressure_solve(ops.projection_rhs(s, L))
        unew, pnew = ops.projection_correct(phi, s, p, True)
        if rec is not None:
            q, _ = ops.projection_correct(phi, s, p, False)
            rec.append((u, outflow_clamp_mask(self.dims, *q)))
        return (unew, u, pnew, c)

    def forward(self, theta, forcing, u0, p0) -> float:
        """J; keeps the checkpoints of this run for gradient()."""
        theta = np.zeros(self.B.shape[0]) if theta is None else np.asarray(theta, dtype=np.float64)
        self.ops.set_inflow(self.u_w0 + theta @ self.B)
        st = self._initial(u0, p0)
        self.checkpoints = {}
        J = 0.0
        for n in range(self.S):
            if n % self.every == 0:
                self.checkpoints[n] = st
            st = self._step(st, forcing)
            J += self.ops.drag(st[0], st[2]) / self.S
        self.final = st
        return J

    # -- reverse -------------------------------------------------------------
    def gradient(self, theta, forcing, u0, p0):
        """(J, dJ/dtheta, dJ/df as three staggered-grid arrays)."""
        ops, src = self.ops, self.src
        J = self.forward(theta, forcing, u0, p0)
        co2 = float(ops.par["coef2"])
        gu, gp = ops.drag_gradient()
        gu = [a / self.S for a in gu]
        gp = gp / self.S
        ub = [np.where(f, a, 0.0) for f, a in zip(self.fluid, gu)]
        upb = [np.zeros_like(a) for a in ub]
        pb = gp.copy()
        pab = [np.zeros_like(a) for a in ub]
        uwb = np.zeros_like(self.u_w0)
        fb = [np.zeros_like(a) for a in ub]
        starts = sorted(self.checkpoints)
        recomputed = 0
        for k in reversed(range(len(starts))):
            n0 = starts[k]
            n1 = starts[k + 1] if k + 1 < len(starts) else self.S
            rec, st = [], self.checkpoints[n0]
            for _ in range(n0, n1):
                st = self._step(st, forcing, rec)
                recomputed += 1
            for n in reversed(range(n0, n1)):
                un, masks = rec[n - n0]
                qb = [np.where(m, 0.0, a) for m, a in zip(masks, ub)]
                sb, Lb = ops.projection_adjoint(qb, pb)
                ub_in = [a.copy() for a in upb]
                cb = [a.copy() for a in pab]
                rs = []
                for d in range(3):
                    rb = ops.helm_solve_T(d, np.where(self.fluid[d], sb[d], 0.0))
                    rb = np.where(self.fluid[d], rb, 0.0)
                    fb[d] += self.fvof[d] * rb
                    ub_in[d] += (-2.0 * co2) * ops.vof[d] * rb
                    upb[d] = (0.5 * co2) * ops.vof[d] * rb
                    pab[d] = -rb
                    cb[d] += 2.0 * rb
                    rs.append(rb)
                uwb += src.helmholtz_flux_T(-rs[0])
                pb = pb - ops.gradient_T(rs)
                for d in range(3):
                    for e, a in enumerate(ops.conv_adjoint(d, un, cb[d])):
                        ub_in[e] += a
                uxb, uzb, w = src.convective_flux_T(cb[2], un[0], un[2])
                ub_in[0] += uxb
                ub_in[2] += uzb
                uwb += w
                uxb, w = src.laplace_flux_T(Lb)
                ub_in[0] += uxb
                uwb += w
                if n >= 1:
                    for d in range(3):
                        ub_in[d] += gu[d]
                    pb = pb + gp
                ub = [np.where(f, a, 0.0) for f, a in zip(self.fluid, ub_in)]
                upb = [np.where(f, a, 0.0) for f, a in zip(self.fluid, upb)]
        # the initial history a^0 = flux2(u^0, u_w) + C(u^0) u^0 reads u_w through flux2_z
        u0v = self.checkpoints[0][0]
        uwb += src.convective_flux_T(pab[2], u0v[0], u0v[2])[2]
        self.stats = {"recomputed_steps": recomputed, "checkpoints": len(starts)}
        return J, self.B @ uwb, fb


class FlowAdjointDevice:
    """FlowAdjoint with the state, the checkpoints, the segment records and
    every cotangent in device memory (torch CUDA tensors as buffers), the
    work done by the *_device entry points on the contexts of a GpuFlowOps:
    the outflow clamps' transpose (lsg_clamp_transpose_device), the boundary
    source terms' transposes as scatter-adds over index sets built once
    (lsg_scatter_add_device) and the cotangent updates (lsg_axpy_device) are
    library kernels too; torch only allocates the buffers.  No host copies
    inside a step except the drag value and the iteration counts.  Same
    arguments and results as FlowAdjoint."""

    def __init__(self, ops: GpuFlowOps, steps: int, every: int = 10, device: int = 0):
        import ctypes
        import torch
        self.torch, self.ct = torch, ctypes
        self.ops = ops
        self.S = int(steps)
        self.every = max(1, int(every))
        N, M, K = self.dims = ops.dims
        self.dev = torch.device("cuda", device)
        self.n = N * M * K
        self.gsize = [int(np.prod(grid_dims(d, self.dims))) for d in range(3)]
        g = ops.g
        T = self._t
        self.side_type = T(g["side_type"], torch.int32)
        self.vib, self.vibyx, self.vibzy = T(g["vib"]), T(g["vibyx"]), T(g["vibzy"])
        self.theta_g, self.delta_g = T(g["theta"]), T(g["delta"])
        self.vof = [T(v) for v in ops.vof]
        self.B = inflow_basis(M, K)
        self.u_w0 = np.asarray(g["u_w"], dtype=np.float64)
        self.bc = np.ascontiguousarray(ops.bc, dtype=np.float64)
        self.bc_lap = np.ascontiguousarray(ops.bc_lap, dtype=np.float64)
        self._index_setup(g["theta"], g["delta"], g["bc"], ops.nu)
        gu, gp = ops.drag_gradient()
        self.gu = [T(a) / self.S for a in gu]
        self.gp = T(gp) / self.S
        self.stats = {}

    def _index_setup(self, theta, delta, bc, nu):
        """Index sets and coefficients of the boundary transposes, as device
        tensors."""
        torch = self.torch
        T = self._t
        N, M, K = self.dims
        src = SourceTermTransposes(self.dims, theta, delta, bc, nu)
        # the boundary source terms' transposes as scatter-adds (dst index,
        # src index, coefficient, optional second factor's index), run by
        # lsg_scatter_add_device
        sc = {"cz_in0": (src.cz_in_w, src.cz_in, src.cz_in_c0, None),
              "cz_in1": (src.cz_in_w + M, src.cz_in, src.cz_in_c1, None),
              "cz_last_u0": (src.cz_last, src.cz_last, 0.25 * src.cz_dz * src.cz_dy, src.cz_u0),
              "cz_last_u1": (src.cz_last, src.cz_last, 0.25 * src.cz_dzz * src.cz_dy, src.cz_u1),
              "cz_u0": (src.cz_u0, src.cz_last, 0.25 * src.cz_dy * src.cz_dz, src.cz_last),
              "cz_u1": (src.cz_u1, src.cz_last, 0.25 * src.cz_dy * src.cz_dzz, src.cz_last),
              "cz_nb": (src.cz_nb, src.cz_nb, src.cz_cb, src.cz_nb),
              "cz_nt": (src.cz_nt, src.cz_nt, src.cz_ct, src.cz_nt),
              "hx": (src.hx_w, src.hx_row, -src.hx_c, None),
              "lap_out": (src.lap_out_u, src.lap_out, src.lap_out_c, None),
              "lap_in": (src.lap_in_w, src.lap_in, src.lap_in_c, None)}
        self.sc = {k: (T(di, torch.int64), T(si, torch.int64), T(c), None if s2 is None else T(s2, torch.int64))
                   for k, (di, si, c, s2) in sc.items()}
        # (smallest index, end of each index set) for the host-side bounds
        # check of every scatter
        rng_ = lambda a: (int(np.min(a)), int(np.max(a)) + 1) if np.size(a) else (0, 0)   # noqa: E731
        self.sc_bounds = {k: (rng_(di), rng_(si), None if s2 is None else rng_(s2))
                          for k, (di, si, c, s2) in sc.items()}

    # -- helpers ---------------------------------------------------------------
    def _t(self, a, dtype=None):
        torch = self.torch
        t = torch.as_tensor(np.ascontiguousarray(a), device=self.dev)
        return t.to(dtype or torch.float64).contiguous()

    def _p(self, t, numel=None):
        """Device pointer of a contiguous float64 (or int32) tensor of the
        expected size on this device."""
        assert t.is_contiguous() and t.device == self.dev
        if numel is not None:
            assert t.numel() == numel, (t.numel(), numel)
        return self.ct.c_void_p(t.data_ptr())

    def _sync(self):
        self.torch.cuda.synchronize(self.dev)

    def _empty(self, n):
        return self.torch.empty(n, dtype=self.torch.float64, device=self.dev)

    def _zeros(self, n):
        return self.torch.zeros(n, dtype=self.torch.float64, device=self.dev)

    def _scatter(self, key, dst, src, src2=None):
        """dst[di] += coef * src[si] (* src2[s2i]) with the index set `key`."""
        pr = self.ops.pres
        di, si, c, s2i = self.sc[key]
        bd, bs, bs2 = self.sc_bounds[key]
        assert bd[0] >= 0 and bd[1] <= dst.numel() and bs[0] >= 0 and bs[1] <= src.numel(), key
        assert (src2 is None) == (s2i is None), key
        assert src2 is None or (bs2[0] >= 0 and bs2[1] <= src2.numel()), key
        pr.ctx.check(pr.ctx.lib.lsg_scatter_add_device(
            pr.ctx.h, di.numel(), self._p(dst), self._p(di), self._p(src), self._p(si), self._p(c),
            None if src2 is None else self._p(src2), None if src2 is None else self._p(s2i)))

    def _axpy(self, alpha, x, y):
        pr = self.ops.pres
        pr.ctx.check(pr.ctx.lib.lsg_axpy_device(pr.ctx.h, y.numel(), float(alpha), self._p(x), self._p(y)))

    def _vel(self, u):
        return [self._p(u[d], self.gsize[d]) for d in range(3)]

    def _solve(self, solver, b, x):
        from . import _lib as L
        st = L.Stats()
        self._sync()
        solver.ctx.check(solver.ctx.lib.lsg_solve_device(solver.ctx.h, self._p(b, x.numel()), self._p(x),
                                                         self.ct.byref(st)))
        self._sync()
        return st.iterations

    # -- forward ---------------------------------------------------------------
    def _set_inflow(self, theta):
        u_w = self.u_w0 if theta is None else self.u_w0 + np.asarray(theta, dtype=np.float64) @ self.B
        self.u_w = self._t(u_w)
        self.ops.set_inflow(u_w)
        self.hflux = [self._t(h) for h in self.ops.hflux]

    def _conv(self, d, u):
        from . import _lib as L
        ops = self.ops
        N, M, K = self.dims
        flux2, out = self._empty(self.gsize[d]), self._empty(self.gsize[d])
        self._sync()
        m = ops.mom[d]
        m.ctx.check(m.ctx.lib.lsg_convective_flux_device(m.ctx.h, d, N, M, K, self._p(self.theta_g, 3 * self.n),
                                                         self._p(self.delta_g, 3 * self.n), *self._vel(u),
                                                         self._p(self.u_w), L.dptr(self.bc), self._p(flux2)))
        pr = ops.pres
        pr.ctx.check(pr.ctx.lib.lsg_convective_apply_device(pr.ctx.h, d, *self._vel(u), self._p(u[d]),
                                                            self._p(flux2), self._p(out), 1))
        self._sync()
        return out

    def _initial(self, u0, p0):
        u = [self._t(a) for a in u0]
        return (u, [a.clone() for a in u], self._t(p0), [self._conv(d, u) for d in range(3)])

    def _step(self, st, forcing, rec=None):
        from . import _lib as L
        ops, par = self.ops, self.ops.par
        pr = ops.pres
        lib = pr.ctx.lib
        u, uprev, p, pa = st
        Lf = self._empty(self.n)
        self._sync()
        pr.ctx.check(lib.lsg_laplace_flux_device(pr.ctx.h, self._p(self.side_type), self._p(self.vib),
                                                 self._p(self.u_w), L.dptr(self.bc_lap), self._p(u[0]), self._p(Lf)))
        s, c = [], []
        for d in range(3):
            cd = self._conv(d, u)
            right, aux, gpw = (self._empty(self.gsize[d]) for _ in range(3))
            pr.ctx.check(lib.lsg_momentum_rhs_device(pr.ctx.h, d, self._p(cd), self._p(u[d]), self._p(uprev[d]),
                                                     self._p(self.vof[d]), self._p(self.hflux[d]),
                                                     self._p(p, self.n), self._p(pa[d]), float(par["coef2"]),
                                                     self._p(right), self._p(aux), self._p(gpw)))
            self._sync()
            if forcing is not None:
                self._axpy(1.0, forcing[d], right)         # forcing[d] = vof-weighted forcing field
            x = u[d].clone()
            self._solve(ops.mom[d], right, x)
            s.append(x)
            c.append(cd)
        b = self._empty(self.n)
        pr.ctx.check(lib.lsg_projection_rhs_device(pr.ctx.h, *self._vel(s), self._p(Lf), self._p(b)))
        phi = self._zeros(self.n)
        self._solve(pr, b, phi)
        unew = [self._empty(n) for n in self.gsize]
        pnew = p.clone()
        pr.ctx.check(lib.lsg_projection_correct_device(pr.ctx.h, self._p(phi), *self._vel(s), *self._vel(unew),
                                                       self._p(pnew, self.n), float(par["coef"]), float(par["vbase"]),
                                                       1))
        if rec is not None:
            q = [self._empty(n) for n in self.gsize]
            pq = p.clone()
            pr.ctx.check(lib.lsg_projection_correct_device(pr.ctx.h, self._p(phi), *self._vel(s), *self._vel(q),
                                                           self._p(pq, self.n), float(par["coef"]),
                                                           float(par["vbase"]), 0))
            self._sync()
            rec.append((u, q))
        self._sync()
        return (unew, u, pnew, c)

    def _drag(self, u, p):
        self._sync()
        r = self.ops.loads.calculate_device(u[0].data_ptr(), u[1].data_ptr(), u[2].data_ptr(), p.data_ptr(),
                                            self.vib.data_ptr(), self.vibyx.data_ptr(), self.vibzy.data_ptr(),
                                            self.ops.nu)
        return float(r.coef[0])

    def _forcing(self, forcing):
        """The forcing field weighted by the fluid faces' volumes (the term the
        momentum right-hand side adds), uploaded once per call."""
        if forcing is None:
            return None
        return [self._t(np.where(np.asarray(f_) != 0, v, 0.0) * np.asarray(f, dtype=np.float64))
                for f_, v, f in zip(self.ops.stypes, self.ops.vof, forcing)]

    def forward(self, theta, forcing, u0, p0) -> float:
        self._set_inflow(theta)
        fr = self._forcing(forcing)
        st = self._initial(u0, p0)
        self.checkpoints = {}
        J = 0.0
        for n in range(self.S):
            if n % self.every == 0:
                self.checkpoints[n] = st
            st = self._step(st, fr)
            J += self._drag(st[0], st[2]) / self.S
        self.final = st
        return J

    # -- reverse ---------------------------------------------------------------
    def _conv_flux_T(self, cbar, ux, uz, ub, uwb):
        """(u_x, u_z, u_w) cotangents of <cbar, flux2_z(u, u_w)> added into
        (ub[0], ub[2], uwb), as SourceTermTransposes.convective_flux_T."""
        self._scatter("cz_in0", uwb, cbar)
        self._scatter("cz_in1", uwb, cbar)
        self._scatter("cz_last_u0", ub[2], cbar, ux)
        self._scatter("cz_last_u1", ub[2], cbar, ux)
        self._scatter("cz_u0", ub[0], cbar, uz)
        self._scatter("cz_u1", ub[0], cbar, uz)
        self._scatter("cz_nb", ub[2], cbar, uz)
        self._scatter("cz_nt", ub[2], cbar, uz)

    def gradient(self, theta, forcing, u0, p0):
        """(J, dJ/dtheta, dJ/df): host numpy results, as FlowAdjoint.gradient."""
        from . import _lib as L
        torch = self.torch
        ops = self.ops
        pr = ops.pres
        lib = pr.ctx.lib
        J = self.forward(theta, forcing, u0, p0)
        fr = self._forcing(forcing)
        co2, coef = float(ops.par["coef2"]), float(ops.par["coef"])
        z = lambda a: torch.zeros_like(a)                                    # noqa: E731
        ub = [self._empty(n) for n in self.gsize]
        for d in range(3):
            pr.ctx.check(lib.lsg_fluid_faces_device(pr.ctx.h, d, self._p(self.gu[d]), self._p(ub[d])))
        upb = [z(a) for a in ub]
        pb = self.gp.clone()
        pab = [z(a) for a in ub]
        uwb = self._zeros(self.u_w0.size)
        fb = [z(a) for a in ub]
        starts = sorted(self.checkpoints)
        recomputed = 0
        for k in reversed(range(len(starts))):
            n0 = starts[k]
            n1 = starts[k + 1] if k + 1 < len(starts) else self.S
            rec, st = [], self.checkpoints[n0]
            for _ in range(n0, n1):
                st = self._step(st, fr, rec)
                recomputed += 1
            for n in reversed(range(n0, n1)):
                un, q = rec[n - n0]
                qb = [self._empty(m) for m in self.gsize]
                pr.ctx.check(lib.lsg_clamp_transpose_device(pr.ctx.h, self._p(q[0]), self._p(q[2]), *self._vel(ub),
                                                            *self._vel(qb)))
                sb = [self._empty(m) for m in self.gsize]
                Lb = self._empty(self.n)
                stt = L.Stats()
                self._sync()
                pr.ctx.check(lib.lsg_projection_adjoint_device(pr.ctx.h, *self._vel(qb), self._p(pb, self.n), coef,
                                                               *self._vel(sb), self._p(Lb), self.ct.byref(stt)))
                ub_in = [a.clone() for a in upb]
                cb = [a.clone() for a in pab]
                rs = []
                for d in range(3):
                    # the momentum equation's transposed solve on its fluid
                    # faces, then the cotangents of its right-hand side's
                    # terms in one library kernel
                    g_ = self._empty(self.gsize[d])
                    pr.ctx.check(lib.lsg_fluid_faces_device(pr.ctx.h, d, self._p(sb[d]), self._p(g_)))
                    rsol = self._zeros(self.gsize[d])
                    self._solve(ops.momT[d], g_, rsol)
                    rb = self._empty(self.gsize[d])
                    pr.ctx.check(lib.lsg_momentum_cotangents_device(
                        pr.ctx.h, d, self._p(self.vof[d]), self._p(rsol), co2, self._p(rb), self._p(fb[d]),
                        self._p(ub_in[d]), self._p(upb[d]), self._p(pab[d]), self._p(cb[d])))
                    rs.append(rb)
                self._scatter("hx", uwb, rs[0])
                gT = self._empty(self.n)
                self._sync()
                pr.ctx.check(lib.lsg_gradient_transpose_device(pr.ctx.h, *self._vel(rs), self._p(gT)))
                self._axpy(-1.0, gT, pb)
                for d in range(3):
                    self._sync()
                    pr.ctx.check(lib.lsg_convective_adjoint_device(pr.ctx.h, d, *self._vel(un), self._p(un[d]),
                                                                   self._p(cb[d], self.gsize[d]),
                                                                   *self._vel(ub_in), self._p(ub_in[d]), 1))
                self._sync()
                self._conv_flux_T(cb[2], un[0], un[2], ub_in, uwb)
                self._scatter("lap_out", ub_in[0], Lb)
                self._scatter("lap_in", uwb, Lb)
                if n >= 1:
                    for d in range(3):
                        self._axpy(1.0, self.gu[d], ub_in[d])
                    self._axpy(1.0, self.gp, pb)
                ub = [self._empty(n) for n in self.gsize]
                for d in range(3):
                    pr.ctx.check(lib.lsg_fluid_faces_device(pr.ctx.h, d, self._p(ub_in[d]), self._p(ub[d])))
                    pr.ctx.check(lib.lsg_fluid_faces_device(pr.ctx.h, d, self._p(upb[d]), self._p(upb[d])))
        u0v = self.checkpoints[0][0]
        tmp = [z(a) for a in u0v]
        self._conv_flux_T(pab[2], u0v[0], u0v[2], tmp, uwb)
        self._sync()
        self.stats = {"recomputed_steps": recomputed, "checkpoints": len(starts)}
        return J, self.B @ uwb.cpu().numpy(), [f.cpu().numpy() for f in fb]
