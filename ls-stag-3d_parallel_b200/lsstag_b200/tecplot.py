"""Tecplot solution files of the reference's SolTecplotPrinter
(Base/TecplotPrinters/sol_tecplot_printer.h), written by the library
(lsg_tecplot_sol_write / lsg_tecplot_sol_async): byte for byte the file the
reference prints for the same state.

    write_sol(path, dims, nodes, geom, u, v, w, p)             # host arrays
    w = SolWriter(solver, nodes, geom)                         # a geometry context
    w.write_async(path, u, v, w, p)   # device tensors: copied, then formatted on a host thread
    w.wait()

geom holds delta, theta, celltype, bc (18 boundary velocities) and u_w (the
inflow profile, or None); flow selects the flow task's planes.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L


def cell_centres(dims, h) -> np.ndarray:
    """Cell-centre coordinates (x, y, z interleaved) of a uniform mesh with
    steps h = (hx, hy, hz): the node array the printer reads."""
    N, M, K = (int(v) for v in dims)
    i = np.arange(N * M * K)
    x, y, z = i % N, (i // N) % M, i // (N * M)
    return np.stack([(x + 0.5) * h[0], (y + 0.5) * h[1], (z + 0.5) * h[2]], axis=1).reshape(-1)


def _geom(dims, nodes, geom):
    n = int(np.prod(dims))
    d = lambda a, size: np.ascontiguousarray(a, dtype=np.float64).reshape(-1)[:size]  # noqa: E731
    out = dict(nodes=d(nodes, 3 * n), delta=d(geom["delta"], 3 * n), theta=d(geom["theta"], 3 * n),
               celltype=np.ascontiguousarray(geom["celltype"], dtype=np.int32).reshape(-1),
               bc=d(geom["bc"], 18),
               u_w=None if geom.get("u_w") is None else d(geom["u_w"], dims[1] * dims[2]))
    for k, size in (("nodes", 3 * n), ("delta", 3 * n), ("theta", 3 * n), ("celltype", n), ("bc", 18)):
        if out[k].size != size:
            raise ValueError(f"{k}: {out[k].size} values, expected {size}")
    return out


def write_sol(path: str, dims, nodes, geom: dict, u, v, w, p, flow: bool = True):
    N, M, K = (int(x) for x in dims)
    g = _geom((N, M, K), nodes, geom)
    sizes = ((N - 1) * M * K, N * (M - 1) * K, N * M * (K - 1), N * M * K)
    arrs = [np.ascontiguousarray(a, dtype=np.float64).reshape(-1) for a in (u, v, w, p)]
    for a, s in zip(arrs, sizes):
        if a.size != s:
            raise ValueError(f"field of {a.size} values, expected {s}")
    lib = L.load()
    rc = lib.lsg_tecplot_sol_write(str(path).encode(), N, M, K, L.dptr(g["nodes"]), L.dptr(g["delta"]),
                                   L.dptr(g["theta"]), L.iptr(g["celltype"]), *(L.dptr(a) for a in arrs),
                                   None if g["u_w"] is None else L.dptr(g["u_w"]), L.dptr(g["bc"]), int(bool(flow)))
    if rc != 0:
        raise L.LsgError(rc, f"lsg_tecplot_sol_write failed for {path}")


class SolWriter:
    """Asynchronous writes on a solver context that holds the base grid's
    geometry (e.g. FlowStepper.pres): the call returns once the fields are
    copied to pinned host memory; the formatting and the file write run on
    a host thread until wait()."""

    def __init__(self, solver, nodes, geom: dict, flow: bool = True):
        self.solver = solver
        self.dims = tuple(int(x) for x in solver.dims)
        self.g = _geom(self.dims, nodes, geom)
        self.flow = bool(flow)

    def write_async(self, path: str, u, v, w, p):
        """u, v, w, p: device tensors (or device pointers as ints) of the
        staggered velocities and the pressure, complete on the device."""
        N, M, K = self.dims
        sizes = ((N - 1) * M * K, N * (M - 1) * K, N * M * (K - 1), N * M * K)
        ptrs = []
        for a, s in zip((u, v, w, p), sizes):
            if hasattr(a, "data_ptr"):
                if a.numel() != s or not a.is_contiguous():
                    raise ValueError(f"field of {a.numel()} values, expected {s} (contiguous)")
                ptrs.append(C.c_void_p(a.data_ptr()))
            else:
                ptrs.append(C.c_void_p(int(a)))
        g = self.g
        ctx = self.solver.ctx
        ctx.check(ctx.lib.lsg_tecplot_sol_async(ctx.h, str(path).encode(), L.dptr(g["nodes"]), L.dptr(g["delta"]),
                                                L.dptr(g["theta"]), L.iptr(g["celltype"]), *ptrs,
                                                None if g["u_w"] is None else L.dptr(g["u_w"]), L.dptr(g["bc"]),
                                                int(self.flow)))

    def wait(self):
        ctx = self.solver.ctx
        rc = ctx.lib.lsg_tecplot_wait(ctx.h)
        if rc != 0:
            raise L.LsgError(rc, "the asynchronous Tecplot write failed")
