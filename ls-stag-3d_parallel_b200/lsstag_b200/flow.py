"""Time steps of the fixed-body flow task with every operator on the GPU:
the counterpart of the reference's TimeSteppingMethodInterface::init/step
(TimeSteppingMethod/time_stepping_method_interface.h:150-214) for a flow past
bodies that do not move.

One step, in the reference's order:
  1. the pressure operator's source term from the current x-velocity
     (pEq.m_A->calcFlux: lsg_laplace_flux);
  2. for u, v, w: the convective operator of the current velocities applied
     from the geometry with its source term (ConvectiveDiscreteOperator*
     recalc: lsg_convective_flux + lsg_convective_apply), the right-hand side
     (HelmholtzDiscreteEquation::recalcRightMember: lsg_momentum_rhs) and the
     ILU(0)-FGMRES solve on the momentum operator assembled from the geometry
     (lsg_set_matrix_helmholtz), started from the current velocity;
  3. the pressure equation: b = D u* + flux (lsg_projection_rhs) and the
     MG-FGMRES solve from 0;
  4. the projection (SetSolutions::correction: lsg_projection_correct).
The state (current and previous velocities, pressure, the Adams-Bashforth
history of each momentum equation) lives on the host between the calls.
"""
from __future__ import annotations

import numpy as np

from . import solver as S


class FlowStepper:
    """geom: the mesh arrays (celltype, xtype, ytype, ztype, side_type, theta,
    alpha, delta, inv_vof, vof_x/y/z, inv_mx/my/mz, dib_en/ws/nb/st,
    inv_dib_ne/tn, vib, vibyx, vibzy, u_w, bc (18 boundary velocities), pins);
    par: nu, coef (1.5/dt), coef2 (1/dt), coef_integr (COEF_INTEGR_TIME), eps
    (absolute), vbase, max_it, restart_mom, restart_p; optional eps_p, an
    absolute tolerance of the pressure solve alone (default eps)."""

    def __init__(self, geom: dict, dims, par: dict, u0, v0, w0, p0, device: int = 0, pressure_mg_fp32: bool = False):
        self.g = geom
        self.dims = tuple(int(v) for v in dims)
        self.par = par
        N, M, K = self.dims
        bc = np.asarray(geom["bc"], dtype=np.float64)
        self.bc = bc
        # U_E, V_S, V_N, W_B, W_T of the pressure equation's source term
        self.bc_lap = bc[[1, 8, 9, 16, 17]].copy()
        ptask = S.Task(eps=par.get("eps_p", par["eps"]), MAX_ITER=int(par["max_it"]),
                       FGMRES_RESTART_NUM=int(par["restart_p"]))
        # pressure: the operator assembled from the geometry (it also serves the
        # projection entry points) solved by MG-FGMRES with the FP64 cycle, as
        # the reference does; or, with pressure_mg_fp32, by MG-FGMRES with the
        # FP32 cycle on the same operator with its pinned rows negated
        # (pins_negated: same solution, a hierarchy without wrong-signed
        # coarse rows, which the FP32 cycle needs)
        from . import _lib as L
        self.pres = S.MGFGMRES(device=device)
        self.pres.set_geometry({k: geom[k] for k in ("celltype", "theta", "delta", "inv_mx", "inv_my", "inv_mz")},
                               self.dims, geom["pins"], task=ptask, setup=not pressure_mg_fp32)
        self.pres.set_staggered_types(geom["xtype"], geom["ytype"], geom["ztype"])
        self.psolve = self.pres
        if pressure_mg_fp32:
            self.psolve = S.MGFGMRES(device=device, mg_precision=L.FP32)
            self.psolve.set_planes(S.pins_negated(self.pres.planes(), geom["pins"]), self.dims, task=ptask)
        mtask = S.Task(eps=par["eps"], MAX_ITER=int(par["max_it"]), FGMRES_RESTART_NUM=int(par["restart_mom"]))
        self.mom, self.hflux = [], []
        for d, c in enumerate("xyz"):
            hg = {k: geom[k] for k in ("theta", "alpha", "delta", "inv_vof", "dib_en", "dib_ws", "dib_nb", "dib_st",
                                       "inv_dib_ne", "inv_dib_tn")}
            hg["stype"] = geom[c + "type"]
            hg["vof"] = geom["vof_" + c]
            s = S.ILUFGMRES(device=device)
            s.set_helmholtz(d, hg, self.dims, par["nu"], par["coef_integr"], True, task=mtask)
            self.mom.append(s)
            self.hflux.append(s.helmholtz_flux(d, self.dims, geom[c + "type"], geom["delta"], geom["u_w"], bc,
                                               par["nu"]))
        self.u = [np.array(a, dtype=np.float64) for a in (u0, v0, w0)]
        self.p = np.array(p0, dtype=np.float64)
        # HelmholtzDiscreteEquation::set: previous velocity = current, history
        # = flux2 + C(u) u of the initial state
        self.uprev = [a.copy() for a in self.u]
        self.pprev = self.p.copy()
        self.prev_aux = [self._convective_term(d) for d in range(3)]
        self.its = None

    def _convective_term(self, d: int) -> np.ndarray:
        g = self.g
        flux2 = self.mom[d].convective_flux(d, self.dims, g["theta"], g["delta"], *self.u, g["u_w"], self.bc)
        return self.pres.convective_apply(d, self.u, self.u[d], init=flux2)

    def step(self):
        g, par = self.g, self.par
        flux_lap = self.pres.laplace_flux(g["side_type"], g["vib"], g["u_w"], self.bc_lap, self.u[0])
        us, its = [], []
        for d, c in enumerate("xyz"):
            aux_in = self._convective_term(d)
            right, aux = self.pres.momentum_rhs(d, None, aux_in, self.u[d], self.uprev[d], g["vof_" + c],
                                                self.hflux[d], self.p, self.prev_aux[d], par["coef2"])
            self.prev_aux[d] = aux
            x = self.u[d].copy()
            its.append(self.mom[d].solve(right, x))
            us.append(x)
        b = self.pres.projection_rhs(us[0], us[1], us[2], flux_lap)
        phi = np.zeros_like(self.p)
        its.append(self.psolve.solve(b, phi))
        self.uprev = [a.copy() for a in self.u]
        self.pprev = self.p.copy()
        p = self.p.copy()
        u, v, w, _ = self.pres.projection_correct(phi, us[0], us[1], us[2], p, par["coef"], par["vbase"])
        self.u = [u, v, w]
        self.p = p
        self.its = its
        self.predictions = us
        self.phi = phi
        return its

    def save_state(self, path: str, it: int, time: float, centers, center_velocities, loads):
        """Write the reference's continue-state file (lsstag_b200.state) for
        this state; centers / center_velocities / loads per immersed body."""
        from .state import FlowState, write_state
        write_state(path, FlowState(int(it), float(time), np.asarray(centers, np.float64).reshape(-1, 3),
                                    np.asarray(center_velocities, np.float64).reshape(-1, 3),
                                    np.asarray(loads, np.float64).reshape(-1, 4),
                                    (self.u[0], self.u[1], self.u[2], self.p),
                                    (self.uprev[0], self.uprev[1], self.uprev[2], self.pprev)))

    @classmethod
    def from_state(cls, geom: dict, dims, par: dict, path: str, n_bodies: int = 1, device: int = 0):
        """Continue from a continue-state file as the reference does
        (TimeSteppingMethodInterface::init with continueSolveTask: the
        equations are set up on the loaded current state, which also becomes
        the previous one).  Returns (stepper, FlowState)."""
        from .state import read_state
        st = read_state(path, dims, n_bodies)
        u, v, w, p = st.current
        return cls(geom, dims, par, u, v, w, p, device=device), st

    def close(self):
        for s in self.mom:
            s.close()
        if self.psolve is not self.pres:
            self.psolve.close()
        self.pres.close()


class FlowStepperNative:
    """The same time step run by the library's native stepper
    (lsg_flow_create / lsg_flow_step, csrc/lsg_flow.cu): C++ drives every
    phase, the three momentum solves run concurrently on host threads of the
    library, the state stays in the stepper's device memory.  Same arguments
    as FlowStepperDevice."""

    def __init__(self, geom: dict, dims, par: dict, u0, v0, w0, p0, device: int = 0, pressure_mg_fp32: bool = False,
                 p_rel_tol: float | None = None):
        import ctypes as C

        from . import _lib as L
        self.C, self.L = C, L
        host = FlowStepper(geom, dims, par, u0, v0, w0, p0, device=device, pressure_mg_fp32=pressure_mg_fp32)
        self.host = host
        self.dims = host.dims
        self.ns = [a.size for a in host.u]
        self.lib = host.pres.ctx.lib
        f8 = lambda a: np.ascontiguousarray(a, dtype=np.float64)  # noqa: E731
        self._keep = {"side_type": np.ascontiguousarray(geom["side_type"], dtype=np.int32), "vib": f8(geom["vib"]),
                      "u_w": f8(geom["u_w"]), "theta": f8(geom["theta"]), "delta": f8(geom["delta"]),
                      "vof": [f8(geom["vof_" + c]) for c in "xyz"], "hflux": [f8(h) for h in host.hflux]}
        k = self._keep
        d = L.FlowDesc()
        d.N, d.M, d.K = self.dims
        d.device = device
        d.pres, d.psolve = host.pres.ctx.h, host.psolve.ctx.h
        for i in range(3):
            d.mom[i] = host.mom[i].ctx.h
            d.vof[i] = k["vof"][i].ctypes.data
            d.hflux[i] = k["hflux"][i].ctypes.data
        d.side_type, d.vib, d.u_w = k["side_type"].ctypes.data, k["vib"].ctypes.data, k["u_w"].ctypes.data
        d.theta, d.delta = k["theta"].ctypes.data, k["delta"].ctypes.data
        for i in range(18):
            d.bc[i] = float(host.bc[i])
        for i in range(5):
            d.bc_lap[i] = float(host.bc_lap[i])
        d.coef, d.coef2, d.vbase = float(par["coef"]), float(par["coef2"]), float(par["vbase"])
        d.p_rel_tol = float(p_rel_tol or 0.0)
        d.zconv_reference = 1
        self.desc = d
        self.h = C.c_void_p()
        rc = self.lib.lsg_flow_create(C.byref(d), C.byref(self.h))
        if rc != L.LSG_OK:
            raise L.LsgError(rc, "lsg_flow_create failed")
        arr3 = C.c_void_p * 3
        u = [f8(a) for a in host.u]
        up = [f8(a) for a in host.uprev]
        aux = [f8(a) for a in host.prev_aux]
        self._check(self.lib.lsg_flow_set_state(self.h, arr3(*[a.ctypes.data for a in u]),
                                                arr3(*[a.ctypes.data for a in up]), f8(host.p).ctypes.data,
                                                arr3(*[a.ctypes.data for a in aux])))

    def _check(self, rc):
        if rc < 0:
            raise self.L.LsgError(rc, self.lib.lsg_flow_last_error(self.h).decode())
        return rc

    def step(self):
        its = (self.C.c_int * 4)()
        self._check(self.lib.lsg_flow_step(self.h, its))
        return list(its)

    def state(self):
        """((u, v, w), p) copied to the host."""
        u = [np.empty(n) for n in self.ns]
        p = np.empty(int(np.prod(self.dims)))
        arr3 = self.C.c_void_p * 3
        self._check(self.lib.lsg_flow_state(self.h, arr3(*[a.ctypes.data for a in u]), p.ctypes.data, None))
        return u, p

    def close(self):
        if self.h:
            self.lib.lsg_flow_destroy(self.h)
            self.h = self.C.c_void_p()
        self.host.close()


class FlowStepperDevice:
    """The same time step with the state and every intermediate vector in
    device memory (torch CUDA tensors as buffers, the library's *_device
    entry points for the work): no host copies inside a step except the
    iteration counts.  Same arguments as FlowStepper."""

    def __init__(self, geom: dict, dims, par: dict, u0, v0, w0, p0, device: int = 0, pressure_mg_fp32: bool = False,
                 p_rel_tol: float | None = None):
        """p_rel_tol: stop each pressure solve at p_rel_tol times the norm of
        its right-hand side (lsg_set_tolerance before the solve) instead of
        the absolute eps."""
        import ctypes as C
        import torch
        self.p_rel_tol = p_rel_tol
        self.torch = torch
        self.C = C
        host = FlowStepper(geom, dims, par, u0, v0, w0, p0, device=device, pressure_mg_fp32=pressure_mg_fp32)
        self.host = host                      # owns the contexts; its first state seeds this one
        self.dims = host.dims
        self.par = par
        dev = torch.device("cuda", device)
        f8 = dict(dtype=torch.float64, device=dev)
        T = lambda a, **kw: torch.as_tensor(np.ascontiguousarray(a), device=dev, **kw).contiguous()  # noqa: E731
        self.side_type = T(geom["side_type"], dtype=torch.int32)
        self.vib = T(geom["vib"], dtype=torch.float64)
        self.u_w = T(geom["u_w"], dtype=torch.float64)
        self.theta = T(geom["theta"], dtype=torch.float64)
        self.delta = T(geom["delta"], dtype=torch.float64)
        self.vof = [T(geom["vof_" + c], dtype=torch.float64) for c in "xyz"]
        self.hflux = [T(h, dtype=torch.float64) for h in host.hflux]
        self.u = [T(a, dtype=torch.float64) for a in host.u]
        self.uprev = [T(a, dtype=torch.float64) for a in host.uprev]
        self.prev_aux = [T(a, dtype=torch.float64) for a in host.prev_aux]
        self.p = T(host.p, dtype=torch.float64)
        n = self.p.numel()
        self.flux_lap = torch.empty(n, **f8)
        self.b = torch.empty(n, **f8)
        self.phi = torch.empty(n, **f8)
        self.us = [torch.empty_like(a) for a in self.u]
        self.unew = [torch.empty_like(a) for a in self.u]
        self.flux2 = [torch.empty_like(a) for a in self.u]
        self.conv = [torch.empty_like(a) for a in self.u]
        self.right = [torch.empty_like(a) for a in self.u]
        self.aux = [torch.empty_like(a) for a in self.u]
        self.gp = [torch.empty_like(a) for a in self.u]
        self.bc = np.ascontiguousarray(host.bc)
        self.bc_lap = np.ascontiguousarray(host.bc_lap)
        self.stats = None
        from concurrent.futures import ThreadPoolExecutor
        self.pool = ThreadPoolExecutor(max_workers=3)
        torch.cuda.synchronize()

    def _p(self, t):
        return self.C.c_void_p(t.data_ptr())

    def step(self):
        from . import _lib as L
        torch, C, par = self.torch, self.C, self.par
        pres, mom = self.host.pres, self.host.mom
        lib = pres.ctx.lib
        N, M, K = self.dims
        ck = pres.ctx.check
        ck(lib.lsg_laplace_flux_device(pres.ctx.h, self._p(self.side_type), self._p(self.vib), self._p(self.u_w),
                                       L.dptr(self.bc_lap), self._p(self.u[0]), self._p(self.flux_lap)))
        for d in range(3):
            m = mom[d]
            m.ctx.check(lib.lsg_convective_flux_device(m.ctx.h, d, N, M, K, self._p(self.theta), self._p(self.delta),
                                                       self._p(self.u[0]), self._p(self.u[1]), self._p(self.u[2]),
                                                       self._p(self.u_w), L.dptr(self.bc), self._p(self.flux2[d])))
            ck(lib.lsg_convective_apply_device(pres.ctx.h, d, self._p(self.u[0]), self._p(self.u[1]),
                                               self._p(self.u[2]), self._p(self.u[d]), self._p(self.flux2[d]),
                                               self._p(self.conv[d]), 1))
            ck(lib.lsg_momentum_rhs_device(pres.ctx.h, d, self._p(self.conv[d]), self._p(self.u[d]),
                                           self._p(self.uprev[d]), self._p(self.vof[d]), self._p(self.hflux[d]),
                                           self._p(self.p), self._p(self.prev_aux[d]), float(par["coef2"]),
                                           self._p(self.right[d]), self._p(self.aux[d]), self._p(self.gp[d])))
            self.prev_aux[d], self.aux[d] = self.aux[d], self.prev_aux[d]
            self.us[d].copy_(self.u[d])
        torch.cuda.synchronize()
        # the three momentum systems are independent given the current state:
        # solved concurrently, each on its own context and stream (the calls
        # release the interpreter lock while they wait on the device)
        stats = [L.Stats() for _ in range(3)]
        futs = [self.pool.submit(lib.lsg_solve_device, mom[d].ctx.h, self._p(self.right[d]), self._p(self.us[d]),
                                 C.byref(stats[d])) for d in range(3)]
        its = []
        for d in range(3):
            mom[d].ctx.check(futs[d].result())
            its.append(stats[d].iterations)
        ck(lib.lsg_projection_rhs_device(pres.ctx.h, self._p(self.us[0]), self._p(self.us[1]), self._p(self.us[2]),
                                         self._p(self.flux_lap), self._p(self.b)))
        self.phi.zero_()
        psolve = self.host.psolve
        if self.p_rel_tol is not None:
            bn = float(torch.linalg.vector_norm(self.b))
            psolve.ctx.check(lib.lsg_set_tolerance(psolve.ctx.h, self.p_rel_tol * bn))
        torch.cuda.synchronize()
        st = L.Stats()
        psolve.ctx.check(lib.lsg_solve_device(psolve.ctx.h, self._p(self.b), self._p(self.phi), C.byref(st)))
        its.append(st.iterations)
        ck(lib.lsg_projection_correct_device(pres.ctx.h, self._p(self.phi), self._p(self.us[0]), self._p(self.us[1]),
                                             self._p(self.us[2]), self._p(self.unew[0]), self._p(self.unew[1]),
                                             self._p(self.unew[2]), self._p(self.p), float(par["coef"]),
                                             float(par["vbase"]), 1))
        # previous <- current, current <- corrected (buffer rotation)
        self.uprev, self.u, self.unew = self.u, self.unew, self.uprev
        return its

    def state(self):
        return [a.cpu().numpy() for a in self.u], self.p.cpu().numpy()

    def close(self):
        self.pool.shutdown()
        self.host.close()
