"""Python mirror of the reference's iterative-solver interface for the
pressure-Poisson system, backed by the B200 C ABI.

The reference drives its solvers through
``IterativeSolverInterface{set(A, b, x, task); solve() -> it; norm_r;
rebuildPreconditioner()}`` (Base/Solvers/iterative_solver_interface.h:31-73)
with the concrete classes ``MGFGMRES`` (Base/Solvers/FGMRES/mg_fgmres.h) and
``ILUBiCGStab`` (Base/Solvers/BiCGStab/ilu_bicgstab.h).  The classes below keep
those names, argument meanings and results: ``set`` takes the operator in the
reference's CSR form plus the task parameters (``eps`` absolute tolerance,
``MAX_ITER``, ``FGMRES_RESTART_NUM``), ``solve`` updates ``x`` in place and
returns the iteration count, and ``norm_r`` / ``it`` hold the final implicit
residual and iteration count.  Errors raise instead of the reference's silent
behaviour; a capped solve is reported through ``status``.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _lib as L


@dataclass
class Task:
    """The task fields the reference's solvers read (base_task_description.h:391-416)."""
    eps: float = 1e-5
    MAX_ITER: int = 200
    FGMRES_RESTART_NUM: int = 30
    n_post: int = 3


def pins_negated(planes: np.ndarray, pins) -> np.ndarray:
    """The seven coefficient planes with the pinned rows negated.  The
    reference pins two rows of the pressure operator to the identity
    (laplace_discrete_operator.h:809-821) while every other row has a
    negative diagonal; the Galerkin hierarchy then holds, in the aggregates
    of the pins, rows whose diagonal is positive or nearly zero next to
    positive off-diagonals, and the line smoother divides by them: the
    cycle's output grows to about 1e4 near a pin on the 128x64x64 sphere
    flow while the solution is O(0.3), more than the FP32 cycle can carry.
    Negated, the pins have the sign of the other rows.  The pressure
    right-hand side is 0 at the pins, so S A x = b has the solution of
    A x = b, and the residual norms are the same (S = diag(+-1))."""
    P = np.array(planes, dtype=np.float64, copy=True)
    for p in pins:
        P[:, int(p)] = -P[:, int(p)]
    return P


class IterativeSolver:
    """Common part of the solver classes (IterativeSolverInterface)."""

    method = L.METHOD_FGMRES
    precond = L.PC_MG

    def __init__(self, device: int = 0, mg_precision: int = L.FP64, zline_reference: bool = True,
                 max_levels: int = 0, omega: float = 0.805, gram_schmidt: int = L.GS_MGS,
                 smoother: int = L.SMOOTHER_ADLJ, n_pre: int = 0, adlj_schedule: int = L.ADLJ_AUTO):
        self.ctx = L.Context(device)
        self.mg_precision = mg_precision
        self.adlj_schedule = adlj_schedule
        self.smoother = smoother
        self.n_pre = n_pre
        self.gram_schmidt = gram_schmidt
        self.zline_reference = zline_reference
        self.max_levels = max_levels
        self.omega = omega
        self.it = 1
        self.norm_r = 0.0
        self.eps = 1e-5
        self.status = L.LSG_OK
        self.stats = L.Stats()
        self._b = None
        self._x = None

    # -- IterativeSolverInterface::set ------------------------------------
    def set(self, A, b: np.ndarray | None = None, x: np.ndarray | None = None, task: Task | None = None,
            setup: bool = True):
        """A = (rowptr, col, val, (N, M, K)) in the reference's CSR layout.
        setup=False stores the operator only (for apply())."""
        rowptr, col, val, dims = A
        task = task or Task()
        self.task = task
        self.eps = float(task.eps)
        self._rowptr = np.ascontiguousarray(rowptr, dtype=np.int32)
        self._col = np.ascontiguousarray(col, dtype=np.int32)
        self._val = np.ascontiguousarray(val, dtype=np.float64)
        self.dims = tuple(int(v) for v in dims)
        N, M, K = self.dims
        self.ctx.check(self.ctx.lib.lsg_set_matrix_csr(self.ctx.h, N, M, K, L.iptr(self._rowptr), L.iptr(self._col),
                                                       L.dptr(self._val)))
        if setup:
            self._setup()
        self._b, self._x = b, x

    def set_planes(self, planes: np.ndarray, dims, task: Task | None = None):
        """Same as set() with the operator as seven coefficient planes
        (b, s, w, p, e, n, t) of shape (7, N*M*K)."""
        self.task = task or Task()
        self.eps = float(self.task.eps)
        self._planes = np.ascontiguousarray(planes, dtype=np.float64)
        self.dims = tuple(int(v) for v in dims)
        N, M, K = self.dims
        self.ctx.check(self.ctx.lib.lsg_set_matrix_stencil7(self.ctx.h, N, M, K, L.dptr(self._planes)))
        self._setup()

    def set_geometry(self, geom: dict, dims, pins, task: Task | None = None, setup: bool = True):
        """Same as set() with the operator assembled on the GPU from the
        cut-cell geometry (celltype, theta, delta, inv_mx, inv_my, inv_mz)."""
        self.task = task or Task()
        self.eps = float(self.task.eps)
        g = {k: np.ascontiguousarray(geom[k], dtype=np.float64) for k in ("theta", "delta", "inv_mx", "inv_my",
                                                                          "inv_mz")}
        ct = np.ascontiguousarray(geom["celltype"], dtype=np.int32)
        self._geom = (g, ct)
        self.dims = tuple(int(v) for v in dims)
        N, M, K = self.dims
        self.ctx.check(self.ctx.lib.lsg_set_matrix_geometry(self.ctx.h, N, M, K, L.iptr(ct), L.dptr(g["theta"]),
                                                            L.dptr(g["delta"]), L.dptr(g["inv_mx"]),
                                                            L.dptr(g["inv_my"]), L.dptr(g["inv_mz"]),
                                                            int(pins[0]), int(pins[1])))
        if setup:
            self._setup()

    def build_mesh(self, dims, h, block, bodies=None, phi=None) -> float:
        """The flow task's mesh build on this context's device
        (lsg_mesh_build): ``bodies`` from lsstag_b200.mesh.bodies_array, or
        ``phi`` the task's own level set at the upper cell corners.  Returns
        the device time in ms."""
        N, M, K = (int(v) for v in dims)
        hh = np.ascontiguousarray(h, dtype=np.float64).reshape(3)
        blk = np.ascontiguousarray(block, dtype=np.int32).reshape(4)
        ms = L.C.c_double(0.0)
        if phi is not None:
            ph = np.ascontiguousarray(phi, dtype=np.float64).reshape(-1)
            rc = self.ctx.lib.lsg_mesh_build(self.ctx.h, N, M, K, L.dptr(hh), L.iptr(blk), 0, None, L.dptr(ph),
                                             L.C.byref(ms))
        else:
            b = np.ascontiguousarray(bodies, dtype=np.float64).reshape(-1)
            rc = self.ctx.lib.lsg_mesh_build(self.ctx.h, N, M, K, L.dptr(hh), L.iptr(blk), b.size // 17, L.dptr(b),
                                             None, L.C.byref(ms))
        self.ctx.check(rc)
        self.mesh_dims = (N, M, K)
        return float(ms.value)

    def mesh_get(self, name: str) -> np.ndarray:
        """One array of the built mesh (names: lsstag_b200.mesh.FIELDS)."""
        from . import mesh as MS
        code, dt, _ = MS.FIELDS[name]
        out = np.empty(MS.field_size(name, self.mesh_dims), dtype=dt)
        self.ctx.check(self.ctx.lib.lsg_mesh_get(self.ctx.h, code, out.ctypes.data_as(L.C.c_void_p)))
        return out

    def set_from_mesh(self, pins, task: Task | None = None, setup: bool = True):
        """Same as set() with the pressure operator assembled on the GPU from
        the mesh this context built (lsg_set_matrix_mesh), pins = the two
        pinned rows; the staggered types for the projection come with it."""
        self.task = task or Task()
        self.eps = float(self.task.eps)
        self.dims = self.mesh_dims
        self.ctx.check(self.ctx.lib.lsg_set_matrix_mesh(self.ctx.h, int(pins[0]), int(pins[1])))
        if setup:
            self._setup()

    def set_helmholtz(self, direction: int, geom: dict, base_dims, nu: float, coef: float, is_flow: bool = True,
                      task: Task | None = None, setup: bool = True):
        """The momentum operator of one direction (HelmholtzDiscreteOperator
        X/Y/Z) assembled on the GPU from the geometry and set as this
        solver's operator.  geom holds stype (the staggered cell types),
        theta, alpha, delta, inv_vof, vof (staggered volumes), dib_en,
        dib_ws, dib_nb, dib_st, inv_dib_ne, inv_dib_tn; base_dims = (N, M, K)."""
        self.task = task or Task()
        self.eps = float(self.task.eps)
        keys = ("theta", "alpha", "delta", "inv_vof", "vof", "dib_en", "dib_ws", "dib_nb", "dib_st", "inv_dib_ne",
                "inv_dib_tn")
        g = {k: np.ascontiguousarray(geom[k], dtype=np.float64).reshape(-1) for k in keys}
        st = np.ascontiguousarray(geom["stype"], dtype=np.int32)
        self._helm = (g, st)
        N, M, K = (int(v) for v in base_dims)
        d = int(direction)
        self.dims = (N - (d == 0), M - (d == 1), K - (d == 2))
        self.ctx.check(self.ctx.lib.lsg_set_matrix_helmholtz(self.ctx.h, d, N, M, K, L.iptr(st),
                                                             *(L.dptr(g[k]) for k in keys), float(nu), float(coef),
                                                             int(bool(is_flow))))
        if setup:
            self._setup()

    def helmholtz_flux(self, direction: int, base_dims, stype, delta, u_w, bc, nu: float, ib_geom: dict | None = None):
        """Source term of the momentum operator of one direction as the
        reference's build() leaves it (inflow, S/N and B/T walls); with
        ib_geom (side_type, theta, alpha, inv_vof, dib_en, dib_ws, dib_nb,
        dib_st, inv_dib_ne, inv_dib_tn, vib, vibyx, vibzy) the immersed-boundary
        term is written over it as the reference does for moving bodies."""
        N, M, K = (int(v) for v in base_dims)
        d = int(direction)
        ns = (N - (d == 0)) * (M - (d == 1)) * (K - (d == 2))
        st = np.ascontiguousarray(stype, dtype=np.int32)
        arr = [np.ascontiguousarray(a, dtype=np.float64).reshape(-1) for a in (delta, u_w, bc)]
        out = np.empty(ns)
        keys = ("theta", "alpha", "inv_vof", "dib_en", "dib_ws", "dib_nb", "dib_st", "inv_dib_ne", "inv_dib_tn",
                "vib", "vibyx", "vibzy")
        if ib_geom is not None:
            sd = np.ascontiguousarray(ib_geom["side_type"], dtype=np.int32)
            gg = [np.ascontiguousarray(ib_geom[k], dtype=np.float64).reshape(-1) for k in keys]
            extra = [L.iptr(sd)] + [L.dptr(a) for a in gg]
        else:
            extra = [None] * 13
        self.ctx.check(self.ctx.lib.lsg_helmholtz_flux(self.ctx.h, d, N, M, K, L.iptr(st), *(L.dptr(a) for a in arr),
                                                       float(nu), int(ib_geom is not None), *extra, L.dptr(out)))
        return out

    def convective_flux(self, direction: int, base_dims, theta, delta, ux, uy, uz, u_w, bc):
        """Source term (flux2) of the convective operator of one direction as
        the reference's time step recomputes it (0 for x and y, as there)."""
        N, M, K = (int(v) for v in base_dims)
        d = int(direction)
        ns = (N - (d == 0)) * (M - (d == 1)) * (K - (d == 2))
        arr = [np.ascontiguousarray(a, dtype=np.float64).reshape(-1) for a in (theta, delta, ux, uy, uz, u_w, bc)]
        out = np.empty(ns)
        self.ctx.check(self.ctx.lib.lsg_convective_flux(self.ctx.h, d, N, M, K, *(L.dptr(a) for a in arr),
                                                        L.dptr(out)))
        return out

    # -- pressure projection (needs set_geometry) -----------------------------
    def set_staggered_types(self, xtype, ytype, ztype):
        self._stypes = tuple(np.ascontiguousarray(t, dtype=np.int32) for t in (xtype, ytype, ztype))
        self.ctx.check(self.ctx.lib.lsg_set_staggered_types(self.ctx.h, *(L.iptr(t) for t in self._stypes)))

    def laplace_flux(self, side_type, vib, u_w, bc, ux) -> np.ndarray:
        """Pressure-equation source term (LaplaceDiscreteOperator flux);
        bc = (U_E, V_S, V_N, W_B, W_T)."""
        st = np.ascontiguousarray(side_type, dtype=np.int32)
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (vib, u_w, bc, ux)]
        f = np.empty(int(np.prod(self.dims)))
        self.ctx.check(self.ctx.lib.lsg_laplace_flux(self.ctx.h, L.iptr(st), *(L.dptr(a) for a in arrs), L.dptr(f)))
        return f

    def convective_apply(self, direction: int, U, v, init=None, zconv_reference: bool = True) -> np.ndarray:
        """init + C(U) v for momentum component direction, C the convective
        operator built from the velocity U = (ux, uy, uz)."""
        us = [np.ascontiguousarray(a, dtype=np.float64) for a in U]
        vv = np.ascontiguousarray(v, dtype=np.float64)
        ii = None if init is None else np.ascontiguousarray(init, dtype=np.float64)
        out = np.empty_like(vv)
        self.ctx.check(self.ctx.lib.lsg_convective_apply(self.ctx.h, int(direction), *(L.dptr(a) for a in us),
                                                         L.dptr(vv), None if ii is None else L.dptr(ii),
                                                         L.dptr(out), int(bool(zconv_reference))))
        return out

    def convective_adjoint(self, direction: int, U, v, lam, zconv_reference: bool = True):
        """(ux_bar, uy_bar, uz_bar, v_bar): gradients of <lam, C(U) v> in the
        three velocity grids and in v."""
        us = [np.ascontiguousarray(a, dtype=np.float64) for a in U]
        vv = np.ascontiguousarray(v, dtype=np.float64)
        ll = np.ascontiguousarray(lam, dtype=np.float64)
        ub = [np.empty_like(a) for a in us]
        vb = np.empty_like(vv)
        self.ctx.check(self.ctx.lib.lsg_convective_adjoint(self.ctx.h, int(direction), *(L.dptr(a) for a in us),
                                                           L.dptr(vv), L.dptr(ll), *(L.dptr(a) for a in ub),
                                                           L.dptr(vb), int(bool(zconv_reference))))
        return ub[0], ub[1], ub[2], vb

    def momentum_rhs(self, direction: int, Cconv, flux2, u, uprev, vof, hflux, p, prev_aux, coef2):
        """(right, aux) of one momentum equation (HelmholtzDiscreteEquation::
        recalcRightMember); Cconv = (rowptr, col, val) of the convective
        operator; aux is the next step's prev_aux.  Cconv = None: flux2
        already holds flux2 + C u (convective_apply with init=flux2)."""
        if Cconv is None:
            csr = (None, None, None)
        else:
            rp = np.ascontiguousarray(Cconv[0], dtype=np.int32)
            col = np.ascontiguousarray(Cconv[1], dtype=np.int32)
            val = np.ascontiguousarray(Cconv[2], dtype=np.float64)
            csr = (L.iptr(rp), L.iptr(col), L.dptr(val))
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (flux2, u, uprev, vof, hflux, p, prev_aux)]
        right = np.empty_like(arrs[1])
        aux = np.empty_like(arrs[1])
        self.ctx.check(self.ctx.lib.lsg_momentum_rhs(self.ctx.h, int(direction), *csr,
                                                     *(L.dptr(a) for a in arrs), float(coef2), L.dptr(right),
                                                     L.dptr(aux)))
        return right, aux

    def projection_rhs(self, u, v, w, flux) -> np.ndarray:
        """b = Dx u + Dy v + Dz w + flux, b[pins] = 0 (recalcRightMember)."""
        args = [np.ascontiguousarray(a, dtype=np.float64) for a in (u, v, w, flux)]
        b = np.empty(int(np.prod(self.dims)))
        self.ctx.check(self.ctx.lib.lsg_projection_rhs(self.ctx.h, *(L.dptr(a) for a in args), L.dptr(b)))
        return b

    def projection_correct(self, phi, us, vs, ws, p, coef, vbase, outflow=True):
        """(u, v, w, p) after SetSolutions::correction; p is updated in place."""
        ins = [np.ascontiguousarray(a, dtype=np.float64) for a in (phi, us, vs, ws)]
        outs = [np.empty_like(a) for a in ins[1:]]
        if not (p.dtype == np.float64 and p.flags.c_contiguous):
            raise ValueError("p must be a C-contiguous float64 array (updated in place)")
        self.ctx.check(self.ctx.lib.lsg_projection_correct(self.ctx.h, *(L.dptr(a) for a in ins),
                                                           *(L.dptr(a) for a in outs), L.dptr(p), float(coef),
                                                           float(vbase), int(bool(outflow))))
        return outs[0], outs[1], outs[2], p

    def projection_adjoint(self, ubar_out, vbar_out, wbar_out, pbar_out, coef):
        """Cotangents (ubar, vbar, wbar, fluxbar, pbar) of the inputs of the
        projection step (outflow clamps off) from those of its outputs."""
        ins = [np.ascontiguousarray(a, dtype=np.float64) for a in (ubar_out, vbar_out, wbar_out, pbar_out)]
        outs = [np.empty_like(a) for a in ins[:3]]
        fb = np.empty_like(ins[3])
        self.adj_stats = L.Stats()
        self.ctx.check(self.ctx.lib.lsg_projection_adjoint(self.ctx.h, *(L.dptr(a) for a in ins), float(coef),
                                                           *(L.dptr(a) for a in outs), L.dptr(fb),
                                                           L.C.byref(self.adj_stats)))
        return outs[0], outs[1], outs[2], fb, ins[3].copy()

    def gradient_transpose(self, gx, gy, gz) -> np.ndarray:
        """Gx^T gx + Gy^T gy + Gz^T gz on the base grid (the transposed
        pressure gradient applied from the geometry)."""
        ins = [np.ascontiguousarray(a, dtype=np.float64) for a in (gx, gy, gz)]
        out = np.empty(int(np.prod(self.dims)))
        self.ctx.check(self.ctx.lib.lsg_gradient_transpose(self.ctx.h, *(L.dptr(a) for a in ins), L.dptr(out)))
        return out

    def planes(self) -> np.ndarray:
        n = int(np.prod(self.dims))
        P = np.empty((7, n))
        self.ctx.check(self.ctx.lib.lsg_get_matrix_stencil7(self.ctx.h, L.dptr(P)))
        return P

    def options(self) -> L.Options:
        return L.default_options(method=self.method, precond=self.precond, mg_precision=self.mg_precision,
                                 restart=int(self.task.FGMRES_RESTART_NUM), max_it=int(self.task.MAX_ITER),
                                 n_post=int(self.task.n_post), eps=float(self.eps),
                                 zline_reference=int(self.zline_reference), max_levels=int(self.max_levels),
                                 omega=float(self.omega), gram_schmidt=int(self.gram_schmidt),
                                 smoother=int(self.smoother), n_pre=int(self.n_pre),
                                 adlj_schedule=int(self.adlj_schedule))

    def _setup(self):
        o = self.options()
        self.ctx.check(self.ctx.lib.lsg_setup(self.ctx.h, L.C.byref(o)))

    # -- IterativeSolverInterface::rebuildPreconditioner -------------------
    def rebuildPreconditioner(self):
        self._setup()

    # -- IterativeSolverInterface::solve -----------------------------------
    def solve(self, b: np.ndarray | None = None, x: np.ndarray | None = None) -> int:
        b = self._b if b is None else b
        x = self._x if x is None else x
        if b is None or x is None:
            raise ValueError("solve needs b and x (given here or to set)")
        bb = np.ascontiguousarray(b, dtype=np.float64)
        if not (x.dtype == np.float64 and x.flags.c_contiguous):
            raise ValueError("x must be a C-contiguous float64 array (updated in place)")
        if self.eps != self.task.eps:
            self._setup()
        rc = self.ctx.check(self.ctx.lib.lsg_solve(self.ctx.h, L.dptr(bb), L.dptr(x), L.C.byref(self.stats)))
        self.status = rc
        self.it = self.stats.iterations
        self.norm_r = self.stats.norm_r
        return self.it

    # -- helpers used by the parity tests -----------------------------------
    def apply(self, x: np.ndarray) -> np.ndarray:
        y = np.empty_like(x, dtype=np.float64)
        self.ctx.check(self.ctx.lib.lsg_apply(self.ctx.h, L.dptr(np.ascontiguousarray(x, dtype=np.float64)),
                                              L.dptr(y)))
        return y

    def setup_times(self):
        """(matrix_ms, setup_ms): wall times of the last operator upload or
        assembly with its row-dictionary build, and of the last setup."""
        a, b = L.C.c_double(), L.C.c_double()
        self.ctx.check(self.ctx.lib.lsg_setup_times(self.ctx.h, L.C.byref(a), L.C.byref(b)))
        return a.value, b.value

    def row_classes(self, level: int = 0):
        """(cls, dict) of multigrid level `level` (0 = the operator): each
        row's index into the table of distinct rows (nclass x noff,
        first-seen order)."""
        nc, no = L.C.c_int(), L.C.c_int()
        self.ctx.check(self.ctx.lib.lsg_row_classes(self.ctx.h, level, None, None, L.C.byref(nc), L.C.byref(no)))
        n = int(np.prod(self.level_dims(level) if level > 0 else self.dims))
        cls = np.empty(n, dtype=np.int32)
        dct = np.empty((nc.value, no.value), dtype=np.float64)
        self.ctx.check(self.ctx.lib.lsg_row_classes(self.ctx.h, level, cls.ctypes.data, dct.ctypes.data,
                                                    L.C.byref(nc), L.C.byref(no)))
        return cls, dct

    def precondition(self, b: np.ndarray) -> np.ndarray:
        x = np.empty(b.size, dtype=np.float64)
        self.ctx.check(self.ctx.lib.lsg_precond_apply(self.ctx.h, L.dptr(np.ascontiguousarray(b, dtype=np.float64)),
                                                      L.dptr(x)))
        return x

    # -- adjoint --------------------------------------------------------------
    def apply_transpose(self, x: np.ndarray) -> np.ndarray:
        y = np.empty(x.size, dtype=np.float64)
        self.ctx.check(self.ctx.lib.lsg_apply_transpose(self.ctx.h, L.dptr(np.ascontiguousarray(x, dtype=np.float64)),
                                                        L.dptr(y)))
        return y

    def solve_adjoint(self, g: np.ndarray, lam: np.ndarray | None = None) -> np.ndarray:
        """lambda with A^T lambda = g (same method/preconditioner on A^T)."""
        lam = np.zeros(g.size) if lam is None else lam
        self.adj_stats = L.Stats()
        self.ctx.check(self.ctx.lib.lsg_solve_adjoint(self.ctx.h, L.dptr(np.ascontiguousarray(g, dtype=np.float64)),
                                                      L.dptr(lam), L.C.byref(self.adj_stats)))
        return lam

    def operator_gradient(self, lam: np.ndarray, x: np.ndarray) -> np.ndarray:
        """dJ/dA over the seven coefficient planes: -lambda_i x_{i+off}."""
        g = np.empty((7, x.size))
        self.ctx.check(self.ctx.lib.lsg_operator_gradient(self.ctx.h, L.dptr(np.ascontiguousarray(lam)),
                                                          L.dptr(np.ascontiguousarray(x)), L.dptr(g)))
        return g

    def num_levels(self) -> int:
        return self.ctx.check(self.ctx.lib.lsg_mg_num_levels(self.ctx.h))

    def level_dims(self, level: int):
        d = np.zeros(3, dtype=np.int32)
        self.ctx.check(self.ctx.lib.lsg_mg_level_dims(self.ctx.h, level, L.iptr(d)))
        return tuple(int(v) for v in d)

    def level_csr(self, level: int):
        nnz = L.C.c_longlong(0)
        self.ctx.check(self.ctx.lib.lsg_mg_level_csr(self.ctx.h, level, None, None, None, L.C.byref(nnz)))
        n = int(np.prod(self.level_dims(level)))
        rp = np.zeros(n + 1, dtype=np.int32)
        col = np.zeros(max(1, nnz.value), dtype=np.int32)
        val = np.zeros(max(1, nnz.value), dtype=np.float64)
        self.ctx.check(self.ctx.lib.lsg_mg_level_csr(self.ctx.h, level, L.iptr(rp), L.iptr(col), L.dptr(val),
                                                     L.C.byref(nnz)))
        return rp, col[: nnz.value], val[: nnz.value]

    def level_tridiag(self, level: int, direction: str):
        n = int(np.prod(self.level_dims(level)))
        c = np.zeros(max(1, n - 1))
        d = np.zeros(n)
        e = np.zeros(max(1, n - 1))
        self.ctx.check(self.ctx.lib.lsg_mg_level_tridiag(self.ctx.h, level, direction.encode(), L.dptr(c), L.dptr(d),
                                                         L.dptr(e)))
        return c[: n - 1], d, e[: n - 1]

    def close(self):
        self.ctx.close()


class MGFGMRES(IterativeSolver):
    """FGMRES with the multigrid preconditioner (mg_fgmres.h:33-52)."""
    method = L.METHOD_FGMRES
    precond = L.PC_MG


class ILUBiCGStab(IterativeSolver):
    """BiCGStab with the ILU(0) preconditioner (ilu_bicgstab.h:33-64)."""
    method = L.METHOD_BICGSTAB
    precond = L.PC_ILU0


class ILUFGMRES(IterativeSolver):
    """FGMRES with the ILU(0) preconditioner (ilu_fgmres.h:33-64)."""
    method = L.METHOD_FGMRES
    precond = L.PC_ILU0
