"""Adjoint of the pressure-projection step (lsg_projection_adjoint) through
the C ABI: the projection (right-hand side, pressure solve, velocity and
pressure update, outflow clamps off) is linear, so its adjoint must satisfy
the dot-product identity <y_bar, F(d)> = <F^T(y_bar), d>; wrapped here as a
torch.autograd.Function, its gradient is checked against central finite
differences (step 1e-6) of the FP64 forward projection."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

CASES = ["sphere16", "spheres4_24"]


def _setup(name):
    from lsstag_b200 import solver as S
    from lsstag_b200 import synth
    g = load_golden(name)
    dims = tuple(int(v) for v in g["dims"])
    mask = synth.connected_fluid(g["A_rowptr"], g["A_col"], g["A_val"], g["pins"])
    s = S.MGFGMRES()
    geom = {k: g[k] for k in ("celltype", "theta", "delta", "inv_mx", "inv_my", "inv_mz")}
    s.set_geometry(geom, dims, g["pins"], task=S.Task(eps=1.0, MAX_ITER=400))
    s.set_staggered_types(g["xtype"], g["ytype"], g["ztype"])
    return g, s, dims, mask.astype(np.float64)


def _forward(s, u, v, w, flux, p, coef):
    """Projection with outflow clamps off; the pressure solve to 1e-13."""
    b = s.projection_rhs(u, v, w, flux)
    nb = np.linalg.norm(b)
    phi = np.zeros_like(b)
    if nb > 0:
        s.eps = 1e-13 * nb
        s.task.eps = s.eps
        s.rebuildPreconditioner()                       # the solver reads eps at set-up
        s.solve(b, phi)
    return s.projection_correct(phi, u, v, w, p.copy(), coef, 1.0, outflow=False)


def _phibar_norm(g, ub, vb, wb, pb, coef):
    """||Gx^T S_x ub + Gy^T S_y vb + Gz^T S_z wb + coef pb||, from the
    reference's gradient operators, to size the adjoint solve's tolerance."""
    import scipy.sparse as sp
    n = pb.size
    acc = coef * pb
    for name, inv, x in (("Gx", g["inv_mx"], ub), ("Gy", g["inv_my"], vb), ("Gz", g["inv_mz"], wb)):
        rp = g[name + "_rowptr"]
        G = sp.csr_matrix((g[name + "_val"], g[name + "_col"], rp), shape=(rp.size - 1, n))
        acc = acc + G.T @ (inv * x)
    return float(np.linalg.norm(acc))


def _set_adjoint_eps(s, g, ub, vb, wb, pb, coef):
    s.eps = 1e-12 * _phibar_norm(g, ub, vb, wb, pb, coef)
    s.task.eps = s.eps
    s.rebuildPreconditioner()


def _random_inputs(g, dims, mask, rng):
    N, M, K = dims
    return (rng.standard_normal((N - 1) * M * K), rng.standard_normal(N * (M - 1) * K),
            rng.standard_normal(N * M * (K - 1)), rng.standard_normal(N * M * K) * mask,
            rng.standard_normal(N * M * K) * mask)


@pytest.mark.parametrize("name", CASES)
def test_projection_adjoint_dot_product(name):
    g, s, dims, mask = _setup(name)
    coef = float(g["proj_coef"][0])
    rng = np.random.default_rng(8)
    d = _random_inputs(g, dims, mask, rng)
    yb = _random_inputs(g, dims, mask, rng)
    yb = (yb[0], yb[1], yb[2], yb[4])                       # cotangents of u, v, w, p
    Fd = _forward(s, d[0], d[1], d[2], d[3], d[4], coef)
    lhs = sum(float(np.dot(a, b)) for a, b in zip(yb, Fd))
    _set_adjoint_eps(s, g, yb[0], yb[1], yb[2], yb[3], coef)
    ub, vb, wb, fb, pb = s.projection_adjoint(yb[0], yb[1], yb[2], yb[3], coef)
    rhs = sum(float(np.dot(a, b)) for a, b in zip((ub, vb, wb, fb, pb), d))
    # both solves stop at a relative residual of 1e-13 / 1e-12; the iterates
    # carry that times the conditioning of the cut-cell Laplacian
    assert abs(lhs - rhs) <= 1e-7 * max(abs(lhs), abs(rhs))
    s.close()


def _autograd_fn(s, g, coef):
    import torch

    class ProjectionStep(torch.autograd.Function):
        @staticmethod
        def forward(ctx, u, v, w, flux, p):
            out = _forward(s, u.numpy(), v.numpy(), w.numpy(), flux.numpy(), p.numpy(), coef)
            return tuple(torch.from_numpy(np.ascontiguousarray(o)) for o in out)

        @staticmethod
        def backward(ctx, ub, vb, wb, pb):
            _set_adjoint_eps(s, g, ub.numpy(), vb.numpy(), wb.numpy(), pb.numpy(), coef)
            gu, gv, gw, gf, gp = s.projection_adjoint(ub.numpy(), vb.numpy(), wb.numpy(), pb.numpy(), coef)
            return tuple(torch.from_numpy(np.ascontiguousarray(t)) for t in (gu, gv, gw, gf, gp))

    return ProjectionStep.apply


@pytest.mark.parametrize("name", CASES)
def test_projection_adjoint_gradient_vs_finite_differences(name):
    """J = sum of weighted outputs; dJ/d(u*, v*, w*, flux, p) from the
    adjoint against central finite differences, step 1e-6, in a random
    direction: relative error <= 1e-6."""
    import torch
    g, s, dims, mask = _setup(name)
    coef = float(g["proj_coef"][0])
    rng = np.random.default_rng(9)
    x0 = _random_inputs(g, dims, mask, rng)
    wts = _random_inputs(g, dims, mask, rng)
    wts = (wts[0], wts[1], wts[2], wts[4])
    fn = _autograd_fn(s, g, coef)
    xs = [torch.tensor(a, dtype=torch.float64, requires_grad=True) for a in x0]
    outs = fn(*xs)
    J = sum((torch.from_numpy(wv) * o).sum() for wv, o in zip(wts, outs))
    J.backward()
    grad = [t.grad.numpy() for t in xs]
    dirs = _random_inputs(g, dims, mask, rng)
    h = 1e-6

    def Jnum(sign):
        xx = [a + sign * h * dd for a, dd in zip(x0, dirs)]
        out = _forward(s, *xx, coef)
        return sum(float(np.dot(wv, o)) for wv, o in zip(wts, out))

    fd = (Jnum(+1) - Jnum(-1)) / (2 * h)
    ad = sum(float(np.dot(gr, dd)) for gr, dd in zip(grad, dirs))
    assert abs(fd - ad) <= 1e-6 * abs(ad)
    s.close()
