"""The discrete adjoint of the flow's time steps (lsstag_b200.flow_adjoint) on
the CPU: its host pieces (source-term transposes, outflow clamp mask, plane
transposes) against the oracle's forward functions, and the whole reverse
sweep run on the oracle's operator set (tests/flow_oracle_ops.py) against
central finite differences of the same forward.  The forward composed by
FlowAdjoint is pinned to the reference's own three steps of the 16^3 sphere
flow first."""
import numpy as np
import pytest

from conftest import load_golden

import lsg_oracle as lo
from flow_oracle_ops import OracleFlowOps, load_adjoint_case, planes_csr
from lsstag_b200 import flow_adjoint as FA


@pytest.fixture(scope="module")
def case():
    geom, dims, par = load_adjoint_case()
    return geom, dims, par, OracleFlowOps(geom, dims, par)


def _u0(geom):
    return [geom["u_0"], geom["v_0"], geom["w_0"]], geom["p_0"]


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("d", [0, 1, 2])
@pytest.mark.parametrize("zref", [True, False])
def test_oracle_convective_adjoint_dot_product(case, d, zref):
    geom, dims, par, _ = case
    N, M, K = dims
    rng = np.random.default_rng(10 + d)
    st = geom["xyz"[d] + "type"]
    U = [geom[k] + 0.1 * rng.standard_normal(geom[k].size) for k in ("u_1", "v_1", "w_1")]
    v, lam, dv = (rng.standard_normal(U[d].size) for _ in range(3))
    dU = [rng.standard_normal(a.size) for a in U]
    Ub, vb = lo.convective_adjoint(d, N, M, K, st, geom["theta"], geom["delta"], U, v, lam, zref)
    lhs = lam @ lo.convective_apply(d, N, M, K, st, geom["theta"], geom["delta"], dU, v, zconv_reference=zref) + \
        lam @ lo.convective_apply(d, N, M, K, st, geom["theta"], geom["delta"], U, dv, zconv_reference=zref)
    rhs = sum(a @ b for a, b in zip(Ub, dU)) + vb @ dv
    assert abs(lhs - rhs) <= 1e-13 * (abs(lhs) + 1e-300) + 1e-15


def test_source_term_transposes(case):
    """<bar, f(x + dx) - f(x - dx)> = 2 <f^T bar, dx> for the affine laplace
    and x-momentum terms and the quadratic z convective term (exact for
    polynomials of degree 2)."""
    geom, dims, par, ops = case
    N, M, K = dims
    bc = np.array(geom["bc"], dtype=np.float64)
    bc[12] = 0.7                                            # W_W: exercise the convective inflow term
    src = FA.SourceTermTransposes(dims, geom["theta"], geom["delta"], bc, par["nu"])
    rng = np.random.default_rng(3)
    nx, nz = (N - 1) * M * K, N * M * (K - 1)
    uw, duw = rng.standard_normal(M * K), rng.standard_normal(M * K)
    ux, dux = rng.standard_normal(nx), rng.standard_normal(nx)
    uy = rng.standard_normal(N * (M - 1) * K)
    uz, duz = rng.standard_normal(nz), rng.standard_normal(nz)
    g = geom

    def lap(w, x):
        return lo.laplace_flux(N, M, K, g["celltype"], g["side_type"], g["theta"], g["delta"], g["vib"], w, bc[1],
                               bc[8], bc[9], bc[16], bc[17], x)

    Lb = rng.standard_normal(N * M * K)
    uxb, uwb = src.laplace_flux_T(Lb)
    lhs = Lb @ (lap(uw + duw, ux + dux) - lap(uw - duw, ux - dux))
    assert abs(lhs - 2 * (uxb @ dux + uwb @ duw)) <= 1e-12 * np.abs(lhs)

    hb = rng.standard_normal(nx)
    hx = lambda w: lo.helmholtz_flux(0, N, M, K, g["xtype"], g["delta"], w, bc, par["nu"])
    lhs = hb @ (hx(uw + duw) - hx(uw - duw))
    assert abs(lhs - 2 * (src.helmholtz_flux_T(hb) @ duw)) <= 1e-12 * np.abs(lhs)
    for d in (0, 1):                                       # no u_w in the y, z operators' terms
        f = lambda w: lo.helmholtz_flux(d + 1, N, M, K, g["yz"[d] + "type"], g["delta"], w, bc, par["nu"])
        assert np.array_equal(f(uw), f(uw + duw))

    cb = rng.standard_normal(nz)
    cz = lambda w, x, z: lo.convective_flux(2, N, M, K, g["theta"], g["delta"], x, uy, z, w, bc)
    uxb, uzb, uwb = src.convective_flux_T(cb, ux, uz)
    lhs = cb @ (cz(uw + duw, ux + dux, uz + duz) - cz(uw - duw, ux - dux, uz - duz))
    assert abs(lhs - 2 * (uxb @ dux + uzb @ duz + uwb @ duw)) <= 1e-12 * np.abs(lhs)


def test_outflow_clamp_mask(case):
    geom, dims, par, ops = case
    N, M, K = dims
    rng = np.random.default_rng(4)
    q = [rng.standard_normal(a.size) for a in (geom["u_1"], geom["v_1"], geom["w_1"])]
    mask = FA.outflow_clamp_mask(dims, *q)
    assert all(m.any() for m in mask)
    zero = np.zeros(N * M * K)
    out = lo.projection_correct(ops.G, ops.inv, zero, q[0], q[1], q[2], zero, 1.0, N, M, K, par["vbase"], True)[:3]
    for d in range(3):
        assert np.array_equal(out[d][~mask[d]], q[d][~mask[d]])
        expect = par["vbase"] if d == 0 else 0.0
        assert np.all(out[d][mask[d]] == expect)


def test_planes_transpose_and_decouple():
    rng = np.random.default_rng(6)
    dims = (7, 5, 4)
    N, M, K = dims
    n = N * M * K
    i = np.arange(n)
    x, y, z = i % N, (i // N) % M, i // (N * M)
    ok = (z > 0, y > 0, x > 0, np.ones(n, bool), x < N - 1, y < M - 1, z < K - 1)
    P = np.where(np.array(ok), rng.standard_normal((7, n)), 0.0)       # zero toward cells off the grid
    full = planes_csr(P, dims).toarray()
    T = FA.planes_transpose(P, dims)
    assert np.array_equal(planes_csr(T, dims).toarray(), full.T)
    solid = rng.random(n) < 0.2
    Dc = planes_csr(FA.planes_decouple(P, dims, solid), dims).toarray()
    keep = ~solid
    assert np.array_equal(Dc[np.ix_(keep, keep)], full[np.ix_(keep, keep)])
    off = Dc - np.diag(np.diag(Dc))
    assert not off[solid].any() and not off[:, solid].any()
    assert np.array_equal(np.diag(Dc), np.diag(full))


def test_forward_matches_reference_steps(case):
    """FlowAdjoint's forward (theta = 0, no forcing; exact solves here)
    against the reference's three time steps: velocities within 1e-9.  The
    pressure is compared on the cells that are neither solid nor empty rows of
    the pressure operator (solid cells hold a decoupled 1e-16 diagonal, two
    cut cells of vanishing fluid volume have empty rows and columns: the
    reference's solver leaves values there that nothing reads), within 1e-6:
    the reference stops the pressure solve at an absolute residual of 1e-11,
    and its iterate differs from the exact solution by up to that residual
    over the operator's smallest singular value (4.6e-5)."""
    geom, dims, par, ops = case
    g = load_golden("flow16_steps")
    fa = FA.FlowAdjoint(ops, 3, every=2)
    u0, p0 = _u0(geom)
    fa.forward(None, None, u0, p0)
    u, _, p, _ = fa.final
    for name, mine in zip("uvw", u):
        assert _rel(mine, g[f"{name}_3"]) <= 1e-9, name
    A = planes_csr(lo.laplace_from_geometry(*dims, g["celltype"], g["theta"], g["delta"], g["inv_mx"], g["inv_my"],
                                            g["inv_mz"], g["pins"]), dims)
    live = np.asarray(abs(A).sum(axis=1)).ravel() != 0
    assert (~live).sum() == 2
    live &= np.asarray(g["celltype"]) != lo.SOLID_CELL
    assert _rel(p[live], g["p_3"][live]) <= 1e-6


def test_gradient_vs_central_differences(case):
    """dJ/dtheta (8 inflow modes) and dJ/df along two random directions,
    J the mean drag coefficient over 4 steps, checkpoints every 2 steps,
    against central differences of the same forward (exact solves) with a
    step of 1e-6: relative agreement 1e-6."""
    geom, dims, par, ops = case
    u0, p0 = _u0(geom)
    fa = FA.FlowAdjoint(ops, 4, every=2)
    rng = np.random.default_rng(5)
    th0 = 0.05 * rng.standard_normal(8)
    f0 = [0.01 * rng.standard_normal(a.size) for a in u0]
    J, gth, gf = fa.gradient(th0, f0, u0, p0)
    assert fa.stats == {"recomputed_steps": 4, "checkpoints": 2}
    assert J == fa.forward(th0, f0, u0, p0)
    h = 1e-6
    scale = np.abs(gth).max()
    for k in range(8):
        e = np.zeros(8)
        e[k] = h
        fd = (fa.forward(th0 + e, f0, u0, p0) - fa.forward(th0 - e, f0, u0, p0)) / (2 * h)
        assert abs(gth[k] - fd) <= 1e-6 * max(abs(fd), 1e-2 * scale), (k, gth[k], fd)
    for _ in range(2):
        dirn = [rng.standard_normal(a.size) for a in u0]
        h2 = 1e-6
        fd = (fa.forward(th0, [a + h2 * b for a, b in zip(f0, dirn)], u0, p0) -
              fa.forward(th0, [a - h2 * b for a, b in zip(f0, dirn)], u0, p0)) / (2 * h2)
        ad = sum(a @ b for a, b in zip(gf, dirn))
        assert abs(ad - fd) <= 1e-6 * abs(fd)
    for d in range(3):
        assert not gf[d][np.asarray(ops.stypes[d]) == 0].any()


def test_checkpoint_interval_does_not_change_the_gradient(case):
    geom, dims, par, ops = case
    u0, p0 = _u0(geom)
    rng = np.random.default_rng(8)
    th0 = 0.05 * rng.standard_normal(8)
    res = []
    for every in (1, 3, 4):
        fa = FA.FlowAdjoint(ops, 4, every=every)
        res.append(fa.gradient(th0, None, u0, p0))
        assert fa.stats["checkpoints"] == -(-4 // every)
    for J, gth, gf in res[1:]:
        assert J == res[0][0]
        assert np.array_equal(gth, res[0][1])
        assert all(np.array_equal(a, b) for a, b in zip(gf, res[0][2]))


def test_inflow_basis():
    B = FA.inflow_basis(6, 5)
    assert B.shape == (8, 30)
    y, z = (np.arange(6) + 0.5) / 6, (np.arange(5) + 0.5) / 5
    for k, (a, b) in enumerate(FA.INFLOW_MODES):
        for j in range(6):
            for i in range(5):
                assert B[k, j + i * 6] == pytest.approx(np.sin(a * np.pi * y[j]) * np.sin(b * np.pi * z[i]), abs=1e-15)
    assert np.linalg.matrix_rank(B) == 8


def test_flow_case_carries_the_drag_inputs():
    """The 128x64x64 case holds LoadsCalculator's inputs for the objective:
    the cut-cell list (cut cells of the mesh only, each once) and its
    immersed-boundary arrays; the oracle's drag gradient on them is finite
    and nonzero."""
    from lsstag_b200 import cases
    g, dims, par, _ = cases.load_flow_case()
    N, M, K = dims
    cells = np.asarray(g["cells"])
    ct = np.asarray(g["celltype"])[cells]
    assert cells.size == np.unique(cells).size > 0
    assert np.all((ct != lo.SOLID_CELL) & (ct != lo.FLUID_CELL))
    assert float(g["fcoef"]) > 0
    gx, gy, gz, gp = lo.loads_adjoint(N, M, K, cells, g["celltype"], g["theta"], g["delta"], g["inv_vof"],
                                      g["dmax"], g["dne"], g["dtn"], (float(g["fcoef"]), 0.0, 0.0), par["nu"])
    tot = sum(np.abs(a).sum() for a in (gx, gy, gz, gp))
    assert np.isfinite(tot) and tot > 0


def test_device_sweep_scatter_sets_match_host(case):
    """FlowAdjointDevice's boundary transposes are scatter-adds
    dst[di] += coef * src[si] (* src2[s2i]) run by lsg_scatter_add_device;
    the index sets it builds, applied here with numpy on the CPU, give
    SourceTermTransposes' laplace, helmholtz and convective flux transposes."""
    import torch
    geom, dims, par, ops = case
    N, M, K = dims
    fd = object.__new__(FA.FlowAdjointDevice)           # the index state only, no contexts
    fd.torch, fd.dev, fd.dims = torch, torch.device("cpu"), dims
    fd.gsize = [int(np.prod(FA.grid_dims(d, dims))) for d in range(3)]
    bc = np.array(geom["bc"], dtype=np.float64)
    bc[12] = 0.7
    fd._index_setup(geom["theta"], geom["delta"], bc, par["nu"])
    src = FA.SourceTermTransposes(dims, geom["theta"], geom["delta"], bc, par["nu"])

    def scatter(key, dst, v, v2=None):
        di, si, c, s2i = (None if t is None else t.numpy() for t in fd.sc[key])
        # every index inside its buffer (the device kernel does no bounds check)
        assert di.min() >= 0 and di.max() < dst.size and si.min() >= 0 and si.max() < v.size, key
        assert (v2 is None) == (s2i is None) and (v2 is None or (s2i.min() >= 0 and s2i.max() < v2.size)), key
        assert di.size == si.size == c.size
        w = c * v[si]
        if v2 is not None:
            w = w * v2[s2i]
        np.add.at(dst, di, w)

    rng = np.random.default_rng(9)
    cb, ux, uz = rng.standard_normal(fd.gsize[2]), rng.standard_normal(fd.gsize[0]), rng.standard_normal(fd.gsize[2])
    uxb, uzb, uwb = np.zeros(fd.gsize[0]), np.zeros(fd.gsize[2]), np.zeros(M * K)
    scatter("cz_in0", uwb, cb)
    scatter("cz_in1", uwb, cb)
    scatter("cz_last_u0", uzb, cb, ux)
    scatter("cz_last_u1", uzb, cb, ux)
    scatter("cz_u0", uxb, cb, uz)
    scatter("cz_u1", uxb, cb, uz)
    scatter("cz_nb", uzb, cb, uz)
    scatter("cz_nt", uzb, cb, uz)
    for a, b in zip((uxb, uzb, uwb), src.convective_flux_T(cb, ux, uz)):
        assert np.allclose(a, b, rtol=1e-13, atol=1e-15)
    Lb = rng.standard_normal(N * M * K)
    lx, lw = np.zeros(fd.gsize[0]), np.zeros(M * K)
    scatter("lap_out", lx, Lb)
    scatter("lap_in", lw, Lb)
    hx_, hw_ = src.laplace_flux_T(Lb)
    assert np.allclose(lx, hx_, rtol=1e-13, atol=1e-15) and np.allclose(lw, hw_, rtol=1e-13, atol=1e-15)
    hb = rng.standard_normal(fd.gsize[0])
    hw = np.zeros(M * K)
    scatter("hx", hw, hb)
    # FlowAdjointDevice subtracts the x-momentum cotangents' flux term
    assert np.allclose(hw, -src.helmholtz_flux_T(hb), rtol=1e-13, atol=1e-15)
