"""Pinned rows of the pressure operator and the FP32 multigrid cycle
(lsstag_b200.solver.pins_negated), on the CPU: negating the two identity
rows leaves the pressure solution unchanged, removes the wrong-signed rows
the Galerkin hierarchy otherwise holds in the pins' aggregates, and lets the
FP32 cycle (emulated, tests/mg_fp32_emulation.py) converge on the
128x64x64 sphere flow's operator, where with the reference's pins it
stalls."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spl

from conftest import load_golden

import lsg_oracle as lo
from flow_oracle_ops import planes_csr
from mg_fp32_emulation import MultiGridFP32
from lsstag_b200 import cases
from lsstag_b200.solver import pins_negated


def test_pins_negated_touches_the_pinned_rows_only():
    rng = np.random.default_rng(1)
    P = rng.standard_normal((7, 60))
    Q = pins_negated(P, [3, 41])
    assert np.array_equal(Q[:, [3, 41]], -P[:, [3, 41]])
    keep = np.setdiff1d(np.arange(60), [3, 41])
    assert np.array_equal(Q[:, keep], P[:, keep])


def test_same_pressure_solution():
    """16^3 sphere flow, the reference's first projection: the solution of
    the system with negated pins equals the reference pins' (exact solves
    on the rows that are not empty)."""
    g = load_golden("flow16_steps")
    dims = tuple(int(v) for v in g["dims"])
    N, M, K = dims
    P = lo.laplace_from_geometry(N, M, K, g["celltype"], g["theta"], g["delta"], g["inv_mx"], g["inv_my"],
                                 g["inv_mz"], g["pins"])
    D = lo.divergence_from_geometry(N, M, K, g["celltype"], g["theta"], g["delta"])
    b = lo.projection_rhs(D, g["us_1"], g["vs_1"], g["ws_1"], g["lflux_1"], g["pins"])
    assert not b[np.asarray(g["pins"])].any()
    sol = []
    for Q in (P, pins_negated(P, g["pins"])):
        A = planes_csr(Q, dims).tocsr()
        live = (A.diagonal() != 0) & (np.asarray(g["celltype"]) != lo.SOLID_CELL)
        x = np.zeros(b.size)
        x[live] = spl.spsolve(A[live][:, live].tocsc(), b[live])
        sol.append(x)
    assert np.linalg.norm(sol[0] - sol[1]) <= 1e-12 * np.linalg.norm(sol[0])


@pytest.fixture(scope="module")
def flow_operator():
    g, dims, par, _ = cases.load_flow_case()
    N, M, K = dims
    P = lo.laplace_from_geometry(N, M, K, g["celltype"], g["theta"], g["delta"], g["inv_mx"], g["inv_my"],
                                 g["inv_mz"], g["pins"])
    return g, dims, P


def _wrong_signed_rows(mg):
    """Rows of the coarse levels whose diagonal is positive or weaker than
    half their largest off-diagonal (the line smoother's pivots); rows of
    aggregates of solid cells, whose entries are O(1e-16), do not count."""
    out = []
    for lv in mg.levels[1:]:
        A = lv.A.tocsr()
        dg = A.diagonal()
        off = abs(A - sp.diags(dg)).tocsr()
        mo = np.asarray(off.max(axis=1).todense()).ravel()
        out.append(int(((dg > -0.5 * mo) & (mo > 1e-12)).sum()))
    return out


def test_hierarchy_signs(flow_operator):
    g, dims, P = flow_operator
    ref = _wrong_signed_rows(lo.MultiGrid(planes_csr(P, dims).tocsr(), dims))
    neg = _wrong_signed_rows(lo.MultiGrid(planes_csr(pins_negated(P, g["pins"]), dims).tocsr(), dims))
    assert ref[:3] == [2, 2, 2]                 # the two pins' aggregates, levels 1-3
    assert sum(neg) == 0


def test_fp32_cycle_converges_with_negated_pins(flow_operator):
    """FGMRES(30) with the emulated FP32 cycle on the flow's operator and a
    right-hand side with a nonzero mean (as the flow's mass imbalance gives):
    with the reference's pins the residual is not even halved in 30
    iterations; with negated pins it drops by 1e3 within 8."""
    g, dims, P = flow_operator
    A = planes_csr(P, dims).tocsr()
    live = np.abs(A.diagonal()) >= 1e-12
    rng = np.random.default_rng(2)
    b = np.where(live, rng.standard_normal(A.shape[0]) * 1e-4 + 1e-9, 0.0)
    b[np.asarray(g["pins"])] = 0.0
    eps = 1e-3 * np.linalg.norm(b)
    x, it, _ = lo.fgmres(A, b, np.zeros_like(b), MultiGridFP32(A, dims).apply, eps, 30, 30)
    assert np.linalg.norm(A @ x - b) > 0.5 * np.linalg.norm(b)
    As = planes_csr(pins_negated(P, g["pins"]), dims).tocsr()
    x, it, _ = lo.fgmres(As, b, np.zeros_like(b), MultiGridFP32(As, dims).apply, eps, 30, 30)
    assert it <= 8
    assert np.linalg.norm(A @ x - b) <= eps * 1.0001
