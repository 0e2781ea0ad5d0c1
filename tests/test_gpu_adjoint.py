"""Hand-written adjoint of the pressure solve, through the C ABI, wrapped as
a torch.autograd.Function here (the harness) and checked against central
finite differences of FP64 direct solves (the oracle side)."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spl

from conftest import load_golden

pytestmark = pytest.mark.gpu

CASES = ["sphere16", "spheres4_24"]


def _setup(name, rel=1e-13):
    import lsg_oracle  # noqa: F401  (oracle package on the path)
    import ref_runner as rr
    from lsstag_b200 import solver as S
    from lsstag_b200 import synth
    g = load_golden(name)
    n = g["b"].size
    dims = tuple(int(v) for v in g["dims"])
    A = sp.csr_matrix((g["A_val"], g["A_col"], g["A_rowptr"]), shape=(n, n))
    P = rr.csr_to_planes(g["A_rowptr"], g["A_col"], g["A_val"], dims)
    mask = synth.connected_fluid(g["A_rowptr"], g["A_col"], g["A_val"], g["pins"])
    s = S.MGFGMRES()
    s.set_planes(P, dims, task=S.Task(eps=rel * np.linalg.norm(g["b"]), MAX_ITER=400))
    return g, A, P, mask, s, dims


@pytest.mark.parametrize("name", CASES)
def test_transpose_apply(name):
    g, A, P, mask, s, dims = _setup(name)
    x = np.random.default_rng(3).standard_normal(A.shape[0])
    y = s.apply_transpose(x)
    ref = A.T @ x
    assert np.linalg.norm(y - ref) <= 1e-14 * np.linalg.norm(ref)
    s.close()


@pytest.mark.parametrize("name", CASES)
def test_adjoint_solve_matches_direct(name):
    g, A, P, mask, s, dims = _setup(name)
    rng = np.random.default_rng(4)
    gv = np.where(mask, rng.standard_normal(A.shape[0]), 0.0)
    s.eps = 1e-12 * np.linalg.norm(gv)
    s.task.eps = s.eps
    s.rebuildPreconditioner()
    lam = s.solve_adjoint(gv)
    S_ = np.nonzero(mask)[0]
    ref = spl.spsolve(A[S_][:, S_].T.tocsc(), gv[S_])     # the connected fluid block
    assert np.linalg.norm(A.T @ lam - gv) <= 1e-10 * np.linalg.norm(gv)
    assert np.linalg.norm(lam[S_] - ref) <= 1e-8 * np.linalg.norm(ref)
    s.close()


def _autograd_fn():
    import torch

    class PoissonSolve(torch.autograd.Function):
        """x = A(planes)^{-1} b with the B200 solver; backward through the
        C-ABI adjoint (A^T lambda = dJ/dx, dJ/db = lambda, dJ/dA = -lambda x^T)."""

        @staticmethod
        def forward(ctx, planes, b, solver):
            x = np.zeros(b.numel())
            solver.solve(b.detach().numpy().astype(np.float64), x)
            ctx.solver = solver
            xt = torch.from_numpy(x)
            ctx.save_for_backward(xt)
            return xt

        @staticmethod
        def backward(ctx, gx):
            (x,) = ctx.saved_tensors
            lam = ctx.solver.solve_adjoint(gx.detach().numpy().astype(np.float64))
            gA = ctx.solver.operator_gradient(lam, x.numpy())
            return torch.from_numpy(gA), torch.from_numpy(lam), None

    return PoissonSolve


@pytest.mark.parametrize("name", CASES)
def test_autograd_gradient_vs_central_differences(name):
    """Directional derivatives of J = w.x(b, A) from the adjoint agree with
    central differences (step 1e-6 relative) of FP64 direct solves to 1e-6."""
    import torch
    g, A, P, mask, s, dims = _setup(name)
    n = A.shape[0]
    rng = np.random.default_rng(5)
    w = np.where(mask, rng.standard_normal(n), 0.0)
    b = g["b"]
    fn = _autograd_fn()
    planes_t = torch.from_numpy(P.copy()).requires_grad_(True)
    b_t = torch.from_numpy(b.copy()).requires_grad_(True)
    x = fn.apply(planes_t, b_t, s)
    J = (torch.from_numpy(w) * x).sum()
    J.backward()
    gb = b_t.grad.numpy()
    gA = planes_t.grad.numpy()

    S_ = np.nonzero(mask)[0]

    def J_direct(bb, AA):
        # FP64 direct solve on the connected fluid block (pins hold 0; solid
        # cells and sealed pockets decouple and carry no right-hand side)
        xs = spl.spsolve(AA[S_][:, S_].tocsc(), bb[S_])
        return float(w[S_] @ xs)

    # direction in b (compatible: on the connected fluid cells)
    db = np.where(mask, rng.standard_normal(n), 0.0)
    h = 1e-6 * np.linalg.norm(b) / np.linalg.norm(db)
    fd = (J_direct(b + h * db, A) - J_direct(b - h * db, A)) / (2 * h)
    ad = float(gb @ db)
    assert abs(ad - fd) <= 1e-6 * abs(fd)
    # direction in the off-diagonal coefficients (existing couplings only)
    import ref_runner as rr
    coo = A.tocoo()
    off = (coo.row != coo.col) & (coo.data != 0.0)
    dvals = np.zeros_like(coo.data)
    dvals[off] = rng.standard_normal(int(off.sum())) * np.abs(coo.data[off])
    D = sp.csr_matrix((dvals, (coo.row, coo.col)), shape=A.shape)
    Dp = rr.csr_to_planes(D.indptr, D.indices, D.data, dims)
    hA = 1e-6
    fdA = (J_direct(b, A + hA * D) - J_direct(b, A - hA * D)) / (2 * hA)
    adA = float(np.sum(gA * Dp))
    assert abs(adA - fdA) <= 1e-6 * abs(fdA)
    s.close()
