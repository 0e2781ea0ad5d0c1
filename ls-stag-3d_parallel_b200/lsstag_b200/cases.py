"""The synthetic pressure-Poisson cases the solver is measured on.

Standalone Poisson solve on the unit cube with four immersed spheres (radii
U[0.05, 0.15], centres U[0.2, 0.8]^3, seeded, see synth.four_spheres) and
homogeneous Neumann walls with the reference's two pinned rows.  Each case
file holds the cut-cell Laplace operator that the reference's own
LaplaceDiscreteOperator assembles for that geometry
(laplace_discrete_operator.h:107-686, fixPoint :809-821), stored as seven
coefficient planes (b, s, w, p, e, n, t) in a compressed .npz; the files are
produced by cases/make_cases.py.  The right-hand side is generated here from
the seed (synth.poisson_rhs).
"""
from __future__ import annotations

import os

import numpy as np

from . import synth

CASE_DIR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "cases")


def case_path(n: int, seed: int = 3) -> str:
    return os.path.join(CASE_DIR, f"spheres4_seed{seed}_{n}.npz")


def planes_to_csr(P: np.ndarray, dims):
    """CSR (rowptr, col, val) with every in-grid neighbour of each row."""
    N, M, K = dims
    n = N * M * K
    NM = N * M
    i = np.arange(n)
    x = i % N
    y = (i // N) % M
    z = i // NM
    offs = [-NM, -N, -1, 0, 1, N, NM]
    ok = [z > 0, y > 0, x > 0, np.ones(n, bool), x < N - 1, y < M - 1, z < K - 1]
    cols = np.stack([np.where(ok[s], i + offs[s], -1) for s in range(7)], axis=1)
    vals = P.T
    mask = cols >= 0
    rowptr = np.concatenate([[0], np.cumsum(mask.sum(axis=1))]).astype(np.int32)
    return rowptr, cols[mask].astype(np.int32), vals[mask].astype(np.float64)


def fluid_mask_from_planes(P: np.ndarray, dims, pins) -> np.ndarray:
    rowptr, col, val = planes_to_csr(P, dims)
    return synth.connected_fluid(rowptr, col, val, pins)


def load(n: int, seed: int = 3):
    """(planes (7, n^3), dims, pins, rhs) of the n^3 four-sphere case."""
    with np.load(case_path(n, seed)) as f:
        P = f["planes"].astype(np.float64)
        dims = tuple(int(v) for v in f["dims"])
        pins = f["pins"].astype(np.int64)
        celltype = f["solid"]
    mask = fluid_mask_from_planes(P, dims, pins)
    # celltype stand-in: solid cells (0) vs the rest (1)
    ct = np.where(celltype, 0, 1)
    b = synth.poisson_rhs(seed, ct, pins, mask)
    return P, dims, pins, b


def build_on_device(n: int, seed: int = 3, device: int = 0):
    """(planes, dims, pins, rhs, mesh_ms) of the n^3 four-sphere case with the
    operator built on the GPU from the seeded spheres alone: the flow task's
    mesh build (lsg_mesh_build) and the Laplace assembly from it
    (lsg_set_matrix_mesh), pins N-1 and NM-1 as in the reference's flow task
    (laplace_discrete_operator.h:809-821).  For the sizes with a case file
    the planes equal the file's, bit for bit."""
    from . import mesh as MS
    from . import solver as S
    dims = (n, n, n)
    h = (1.0 / n,) * 3
    sph = synth.four_spheres(seed)
    pins = np.array([n - 1, n * n - 1], dtype=np.int64)
    s = S.MGFGMRES(device=device)
    try:
        ms = s.build_mesh(dims, h, MS.flow_block(dims, h, sph), bodies=MS.bodies_array(sph))
        s.set_from_mesh(pins, setup=False)
        P = s.planes()
        solid = s.mesh_get("celltype") == 0
    finally:
        s.close()
    mask = fluid_mask_from_planes(P, dims, pins)
    b = synth.poisson_rhs(seed, np.where(solid, 0, 1), pins, mask)
    return P, dims, pins, b, ms


# --------------------------------------------------------------------------
# Flow past a sphere (the plain FP64 LS-STAG flow case): every mesh array of
# the time step, stored sparsely (most frequent value + exceptions) by
# cases/make_flow_case.py
# --------------------------------------------------------------------------
def flow_case_path() -> str:
    return os.path.join(CASE_DIR, "flow_sphere_128x64x64.npz")


def load_flow_case(path: str | None = None):
    """(mesh arrays, dims, params, (u0, v0, w0, p0)) of the flow case, in the
    form lsstag_b200.flow.FlowStepper takes them."""
    z = np.load(path or flow_case_path())
    g = {}
    for k in z.files:
        if k.endswith("__mode"):
            name = k[:-6]
            a = np.full(int(z[name + "__n"]), z[k], dtype=z[k].dtype)
            a[z[name + "__idx"]] = z[name + "__val"]
            g[name] = a
        elif "__" not in k:
            g[k] = z[k]
    nu, coef, coef2, integr, dt, eps, vbase, maxit = (float(v) for v in g["nu_coef_coef2_integr_dt_eps_vbase_maxit"])
    par = dict(nu=nu, coef=coef, coef2=coef2, coef_integr=integr, dt=dt, eps=eps, vbase=vbase, max_it=int(maxit),
               restart_mom=int(g["restart_mom_p"][0]), restart_p=int(g["restart_mom_p"][1]))
    return g, tuple(int(v) for v in g["dims"]), par, (g["u_0"], g["v_0"], g["w_0"], g["p_0"])


def flow_case_on_device(dims, h, spheres=(), ellipsoids=(), Re: float = 100.0, dt: float = 0.01,
                        eps: float = 1e-5, restart_p: int = 30, restart_mom: int = 13, max_it: int = 200,
                        device: int = 0):
    """(mesh arrays, dims, params, (u0, v0, w0, p0)) of a flow past fixed
    bodies on a uniform grid, in the form load_flow_case returns them, with
    the whole mesh built on the GPU from the bodies (lsg_mesh_build) instead of
    read from a case file.  The rest is the reference's flow task set-up:
    uniform inflow U_W = V_BASE = 1 (base_task_description.h:313-315),
    N/S walls u = 1 and W/E u = 1 (flow_task_description.h:79-96), every other
    boundary velocity 0, immersed-boundary velocities 0 (fixed bodies), the
    pinned rows N - 1 and N M - 1 (laplace_discrete_operator.h:809-821), the
    initial state u = 1 on the x-grid cells that are not solid, v = w = p = 0,
    nu = 1 / Re, the BDF2 coefficients 1.5 / dt and 1 / dt.  The loads inputs
    of the drag objective (cut-cell list in the reference's order, delta_ib_max,
    inverse immersed-boundary distances, fcoef = 2) come with it."""
    from . import mesh as MS
    from . import solver as S
    N, M, K = (int(v) for v in dims)
    s = S.MGFGMRES(device=device)
    try:
        s.build_mesh((N, M, K), h, MS.flow_block((N, M, K), h, spheres, ellipsoids),
                     bodies=MS.bodies_array(spheres, ellipsoids))
        g = {k: s.mesh_get(k) for k in ("celltype", "xtype", "ytype", "ztype", "side_type", "theta", "alpha",
                                         "delta", "inv_vof", "vof_x", "vof_y", "vof_z", "inv_mx", "inv_my",
                                         "inv_mz", "dib_en", "dib_ws", "dib_nb", "dib_st", "inv_dib_ne",
                                         "inv_dib_tn", "dib_max")}
    finally:
        s.close()
    n = N * M * K
    g["dims"] = np.array([N, M, K], dtype=np.int32)
    for k in ("vib", "vibyx", "vibzy"):
        g[k] = np.zeros(3 * n)
    g["u_w"] = np.ones(M * K)
    bc = np.zeros(18)
    bc[[0, 1, 2, 3]] = 1.0          # U_W, U_E, U_S, U_N
    g["bc"] = bc
    g["pins"] = np.array([N - 1, N * M - 1], dtype=np.int32)
    ct = g["celltype"]
    g["cells"] = np.nonzero((ct > 0) & (ct < 11111111))[0].astype(np.int32)
    g["dmax"], g["dne"], g["dtn"] = g["dib_max"], g["inv_dib_ne"], g["inv_dib_tn"]
    g["fcoef"] = np.array(2.0)
    par = dict(nu=1.0 / Re, coef=1.5 / dt, coef2=1.0 / dt, coef_integr=1.5 / dt, dt=dt, eps=eps, vbase=1.0,
               max_it=int(max_it), restart_mom=int(restart_mom), restart_p=int(restart_p))
    u0 = np.where(g["xtype"] != 0, 1.0, 0.0)
    v0 = np.zeros(N * (M - 1) * K)
    w0 = np.zeros(N * M * (K - 1))
    p0 = np.zeros(n)
    return g, (N, M, K), par, (u0, v0, w0, p0)
