"""Aerodynamic loads on the immersed boundary, computed on the GPU through the
C ABI (lsg_loads_*): the counterpart of the reference's LoadsCalculator
(Base/loads_calculator.h).

    lc = LoadsCalculator()
    lc.set(dims, cells, celltype, theta, delta, inv_vof, delta_ib_max,
           inv_delta_ib_ne, inv_delta_ib_tn, nodes, center, fcoef, dt)   # set() + the OnAirfoil list
    lc.calculate(ux, uy, uz, p, vib, vib_yx, vib_zy, nu)                # calculate()
    lc.C_d, lc.F_aer_x, lc.moment_aer, lc.ForceX ...

Attribute names follow the reference's public members.  Arrays are numpy
(host) arrays, or device pointers (ints) for calculate_device().
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L


class LoadsCalculator:
    def __init__(self, device: int = 0):
        self.ctx = L.Context(device)
        self.countCutCells = 0
        self.ForceX = self.ForceY = self.ForceZ = np.zeros(0)
        self.F_aer_x = self.F_aer_y = self.F_aer_z = 0.0
        self.C_d = self.C_y = self.C_z = 0.0
        self.moment_aer = self.moment_x_aer = self.moment_y_aer = 0.0
        self.moment_raw = (0.0, 0.0, 0.0)

    def set(self, dims, cells, celltype, theta, delta, inv_vof, delta_ib_max, inv_delta_ib_ne,
            inv_delta_ib_tn, nodes, center, fcoef: float, dt: float):
        """Cut-cell list (base-grid indices, reporting order) and the geometry
        the loads read; coordinate arrays are xyz-interleaved (3n)."""
        N, M, K = (int(v) for v in dims)
        self.dims = (N, M, K)
        ints = [np.ascontiguousarray(a, dtype=np.int32) for a in (cells, celltype)]
        dbl = [np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
               for a in (theta, delta, inv_vof, delta_ib_max, inv_delta_ib_ne, inv_delta_ib_tn, nodes, center)]
        self.countCutCells = int(ints[0].size)
        self.ctx.check(self.ctx.lib.lsg_loads_set(self.ctx.h, N, M, K, self.countCutCells, L.iptr(ints[0]),
                                                  L.iptr(ints[1]), *(L.dptr(a) for a in dbl), float(fcoef),
                                                  float(dt)))

    def _store(self, r: L.LoadsResult):
        self.F_aer_x, self.F_aer_y, self.F_aer_z = r.force
        self.C_d, self.C_y, self.C_z = r.coef
        self.moment_aer, self.moment_x_aer, self.moment_y_aer = r.moment
        self.moment_raw = tuple(r.moment_raw)

    def calculate(self, ux, uy, uz, p, vib, vib_yx, vib_zy, nu: float, nu_cell=None):
        """Per-cut-cell forces (ForceX/Y/Z), their sums, coefficients and the
        filtered moments."""
        arrs = [np.ascontiguousarray(a, dtype=np.float64).reshape(-1) for a in (ux, uy, uz, p, vib, vib_yx, vib_zy)]
        nc = None if nu_cell is None else np.ascontiguousarray(nu_cell, dtype=np.float64)
        forces = np.empty(3 * self.countCutCells)
        r = L.LoadsResult()
        self.ctx.check(self.ctx.lib.lsg_loads_calculate(self.ctx.h, *(L.dptr(a) for a in arrs),
                                                        None if nc is None else L.dptr(nc), float(nu),
                                                        L.dptr(forces), C.byref(r)))
        c = self.countCutCells
        self.ForceX, self.ForceY, self.ForceZ = forces[:c], forces[c:2 * c], forces[2 * c:]
        self._store(r)
        return r

    def calculate_device(self, ux, uy, uz, p, vib, vib_yx, vib_zy, nu: float, nu_cell=0, forces=0):
        """Same on device pointers (ints, e.g. tensor.data_ptr()); forces (3 *
        count doubles on the device) may be 0."""
        r = L.LoadsResult()
        self.ctx.check(self.ctx.lib.lsg_loads_calculate_device(
            self.ctx.h, *(C.c_void_p(int(a)) for a in (ux, uy, uz, p, vib, vib_yx, vib_zy, nu_cell)), float(nu),
            C.c_void_p(int(forces)), C.byref(r)))
        self._store(r)
        return r

    def reset_filter(self, dt: float):
        self.ctx.check(self.ctx.lib.lsg_loads_reset_filter(self.ctx.h, float(dt)))

    def adjoint(self, weight, nu: float, nu_cell=None):
        """(g_ux, g_uy, g_uz, g_p): gradient of weight . (F_aer_x, F_aer_y, F_aer_z)."""
        N, M, K = self.dims
        w = np.ascontiguousarray(weight, dtype=np.float64)
        nc = None if nu_cell is None else np.ascontiguousarray(nu_cell, dtype=np.float64)
        out = [np.empty((N - 1) * M * K), np.empty(N * (M - 1) * K), np.empty(N * M * (K - 1)), np.empty(N * M * K)]
        self.ctx.check(self.ctx.lib.lsg_loads_adjoint(self.ctx.h, L.dptr(w), None if nc is None else L.dptr(nc),
                                                      float(nu), *(L.dptr(a) for a in out)))
        return tuple(out)

    def adjoint_device(self, weight, nu: float, g_ux, g_uy, g_uz, g_p, nu_cell=0):
        w = np.ascontiguousarray(weight, dtype=np.float64)
        self.ctx.check(self.ctx.lib.lsg_loads_adjoint_device(
            self.ctx.h, L.dptr(w), C.c_void_p(int(nu_cell)), float(nu),
            *(C.c_void_p(int(a)) for a in (g_ux, g_uy, g_uz, g_p))))

    def close(self):
        self.ctx.close()
