"""The even-odd-* transfer class, where the product departs from the
reference on purpose.

On a 12 x 10 x 8 grid the first coarsening (12 x 10 x 8 -> 6 x 5 x 4) is
even-even-even and the second (6 x 5 x 4 -> 3 x 3 x 2) even-odd-even.  The
reference's even-odd-* builders (Base/CoarseGrid/TransferOperators/
transfer_operators_even_odd_*.h) give the right weights but point some
entries of the upper z-plane at the wrong coarse cells; the product uses
the tensor product of the 1-D factors those builders are meant to produce
(lsg_oracle.prolong_1d).  Pinned here (fixture tests/golden/mixed12x10x8.npz,
made by tests/golden/make_mixed_parity_golden.py from the reference itself):
  * the first coarsening's P and R equal the reference's bit for bit;
  * the second's P differs from the reference's in exactly the rows whose
    stencil reaches the upper coarse z-plane, with the same weights, and only
    the reference's entries leave the 2x2x2 coarse neighbourhood of the fine
    cell;
  * the CPU restatement with the reference's P substituted reproduces the
    reference's V-cycle and MG-FGMRES solve, so P is the only departure;
  * with the tensor-product P the solve takes the same iteration count, and
    (GPU) the product's V-cycle and solve equal that restatement's."""
import numpy as np
import pytest
import scipy.sparse as sp

import lsg_oracle as lo
from conftest import load_golden


def _csr(g, key, shape):
    return sp.csr_matrix((g[key + "_val"], g[key + "_col"], g[key + "_rowptr"]), shape=shape)


@pytest.fixture(scope="module")
def case():
    g = load_golden("mixed12x10x8")
    n = g["b"].size
    A = sp.csr_matrix((g["A_val"], g["A_col"], g["A_rowptr"]), shape=(n, n))
    dims = tuple(int(v) for v in g["dims"])
    return g, A, dims


def _xyz(i, N, M):
    return i % N, (i // N) % M, i // (N * M)


def test_even_even_even_transfers_equal_reference(case):
    g, A, dims = case
    mg = lo.MultiGrid(A, dims)
    assert len(mg.levels) == 3
    P, R = mg.levels[0].P, mg.levels[0].R
    assert abs(P - _csr(g, "mg0_P", P.shape)).max() == 0.0
    assert abs(R - _csr(g, "mg0_R", R.shape)).max() == 0.0


def test_even_odd_even_departure(case):
    g, A, dims = case
    mg = lo.MultiGrid(A, dims)
    f, c = mg.levels[1], mg.levels[2]
    assert (f.N, f.M, f.K, c.N, c.M, c.K) == (6, 5, 4, 3, 3, 2)
    P = mg.levels[1].P.tocsr()
    Pr = _csr(g, "mg1_P", P.shape).tocsr()
    differ = np.nonzero(np.abs(P - Pr).sum(axis=1).A.ravel() > 0)[0]
    assert differ.size == 36
    for i in range(P.shape[0]):
        mine = P[i].toarray().ravel()
        ref = Pr[i].toarray().ravel()
        # the same weights (and row sum 1) in every row
        assert np.array_equal(np.sort(mine[mine != 0]), np.sort(ref[ref != 0]))
        assert mine.sum() == 1.0
        fx, fy, fz = _xyz(i, f.N, f.M)

        def local(row):
            for j in np.nonzero(row)[0]:
                cx, cy, cz = _xyz(j, c.N, c.M)
                # even dimension: coarse cells (f-1)//2 .. (f+1)//2; odd: f//2 .. (f+1)//2
                if not ((fx - 1) // 2 <= cx <= (fx + 1) // 2 and fy // 2 <= cy <= (fy + 1) // 2
                        and (fz - 1) // 2 <= cz <= (fz + 1) // 2):
                    return False
            return True
        assert local(mine)
        assert local(ref) == (i not in set(differ))


def test_reference_transfer_substituted_reproduces_reference(case):
    g, A, dims = case
    Pr = _csr(g, "mg1_P", (120, 18))
    Rr = _csr(g, "mg1_R", (18, 120))
    assert abs(Rr - Pr.T).max() == 0.0                      # R = P^T in this class
    mg = lo.MultiGrid(A, dims, transfers={1: (Pr, Rr)})
    for l in range(2):
        AH = mg.levels[l + 1].A
        Ar = _csr(g, f"mg{l}_AH", AH.shape)
        assert abs(AH - Ar).max() <= 1e-13 * abs(Ar).max()
    x = mg.apply(g["b"])
    assert np.linalg.norm(x - g["vcycle_x"]) <= 1e-12 * np.linalg.norm(g["vcycle_x"])
    eps = float(g["eps"][0])
    xs, it, _ = lo.fgmres(A, g["b"], np.zeros_like(g["b"]), mg.apply, eps, 30, 200)
    assert it == int(g["fgmres_it"][0])
    assert np.linalg.norm(xs - g["fgmres_x"]) <= 1e-10 * np.linalg.norm(g["fgmres_x"])


def test_tensor_product_transfer_same_iterations(case):
    g, A, dims = case
    mg = lo.MultiGrid(A, dims)
    eps = float(g["eps"][0])
    xs, it, _ = lo.fgmres(A, g["b"], np.zeros_like(g["b"]), mg.apply, eps, 30, 200)
    assert it == int(g["fgmres_it"][0])
    assert np.linalg.norm(A @ xs - g["b"]) <= eps


@pytest.mark.gpu
def test_gpu_cycle_and_solve_follow_tensor_product(case):
    from lsstag_b200 import _lib as L
    from lsstag_b200 import solver as S
    g, A, dims = case
    mg = lo.MultiGrid(A, dims)
    eps = float(g["eps"][0])
    s = S.MGFGMRES(mg_precision=L.FP64)
    s.set((g["A_rowptr"], g["A_col"], g["A_val"], dims), task=S.Task(eps=eps))
    x = s.precondition(g["b"])
    xo = mg.apply(g["b"])
    assert np.linalg.norm(x - xo) <= 1e-12 * np.linalg.norm(xo)
    xs = np.zeros(g["b"].size)
    it = s.solve(g["b"], xs)
    xr, ito, _ = lo.fgmres(A, g["b"], np.zeros_like(g["b"]), mg.apply, eps, 30, 200)
    assert abs(it - ito) <= 1
    assert np.linalg.norm(xs - xr) <= 1e-8 * np.linalg.norm(xr)
    s.close()
