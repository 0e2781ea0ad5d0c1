"""Failure detection of the solver entry points, every failure made on the
host (bad inputs, a call out of order, an iteration cap), plus the bounded
waits of the device code: a wait that runs out (a barrier arrival nobody
makes) ends its kernel with an error flag the host reports.  Nothing here
faults or hangs the GPU, and the context stays usable after each one.

The reference reports none of these: a capped solve returns silently after
MAX_ITER (base_task_description.h:45, fgmres_interface.h:123), NaNs run to
the cap, and the coarsest LU clamps pivots to 1e-13 max|A|
(lu_decomposition_sparse_matrix.h:112, :133, :205) so only an all-zero or
non-finite coarsest matrix has no factorisation."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def _csr(g):
    return (g["A_rowptr"], g["A_col"], g["A_val"], tuple(int(v) for v in g["dims"]))


@pytest.mark.parametrize("cls", ["MGFGMRES", "ILUBiCGStab", "ILUFGMRES"])
def test_nan_in_rhs_is_a_breakdown(cls):
    from lsstag_b200 import _lib as L
    from lsstag_b200 import solver as S
    g = load_golden("sphere16")
    s = getattr(S, cls)()
    s.set(_csr(g), task=S.Task(eps=float(g["eps"][0])))
    b = g["b"].copy()
    b[b.size // 2] = np.nan
    x = np.zeros(b.size)
    s.solve(b, x)
    assert s.status == L.LSG_BREAKDOWN and s.stats.status == L.LSG_BREAKDOWN
    # the context is still usable: the clean system solves
    x = np.zeros(b.size)
    s.solve(g["b"], x)
    assert s.status == L.LSG_OK and np.all(np.isfinite(x))
    s.close()


def test_inf_in_initial_guess_is_a_breakdown():
    from lsstag_b200 import _lib as L
    from lsstag_b200 import solver as S
    g = load_golden("sphere16")
    s = S.MGFGMRES()
    s.set(_csr(g), task=S.Task(eps=float(g["eps"][0])))
    x = np.zeros(g["b"].size)
    x[3] = np.inf
    s.solve(g["b"], x)
    assert s.status == L.LSG_BREAKDOWN
    s.close()


@pytest.mark.parametrize("cls", ["MGFGMRES", "ILUBiCGStab"])
def test_iteration_cap_is_reported(cls):
    from lsstag_b200 import _lib as L
    from lsstag_b200 import solver as S
    g = load_golden("sphere16")
    s = getattr(S, cls)()
    s.set(_csr(g), task=S.Task(eps=float(g["eps"][0]), MAX_ITER=1))
    x = np.zeros(g["b"].size)
    it = s.solve(g["b"], x)
    # the reference's counting: FGMRES counts inner steps from 1, BiCGStab
    # starts its counter at 1 and increments after each pass
    # (bicgstab_interface.h:76-111), so one pass reports 2
    assert it == (1 if cls == "MGFGMRES" else 2)
    assert s.status == L.LSG_NOT_CONVERGED and s.stats.status == L.LSG_NOT_CONVERGED
    assert s.norm_r > float(g["eps"][0])
    s.close()


def test_zero_operator_has_no_coarse_factorisation():
    from lsstag_b200 import _lib as L
    from lsstag_b200 import solver as S
    g = load_golden("sphere16")
    dims = tuple(int(v) for v in g["dims"])
    s = S.MGFGMRES()
    with pytest.raises(L.LsgError) as e:
        s.set_planes(np.zeros((7, int(np.prod(dims)))), dims)
    assert e.value.code == L.LSG_ERR_SINGULAR
    # a NaN coefficient reaches the coarsest level through the Galerkin products
    P = np.zeros((7, int(np.prod(dims))))
    P[3] = -1.0
    P[3, 100] = np.nan
    with pytest.raises(L.LsgError) as e:
        s.set_planes(P, dims)
    assert e.value.code == L.LSG_ERR_SINGULAR
    s.close()


def test_calls_out_of_order():
    import ctypes

    from lsstag_b200 import _lib as L
    from lsstag_b200 import solver as S
    g = load_golden("sphere16")
    n = g["b"].size
    ctx = L.Context(0)
    lib = ctx.lib
    st = L.Stats()
    b = np.ascontiguousarray(g["b"])
    x = np.zeros(n)
    # no operator, no setup
    assert lib.lsg_solve(ctx.h, L.dptr(b), L.dptr(x), ctypes.byref(st)) == L.LSG_ERR_STATE
    o = L.default_options()
    assert lib.lsg_setup(ctx.h, ctypes.byref(o)) == L.LSG_ERR_STATE
    assert "lsg_set_matrix_csr" in lib.lsg_last_error(ctx.h).decode()
    # operator set, setup missing
    rp, col, val = (np.ascontiguousarray(g[k]) for k in ("A_rowptr", "A_col", "A_val"))
    N, M, K = (int(v) for v in g["dims"])
    ctx.check(lib.lsg_set_matrix_csr(ctx.h, N, M, K, L.iptr(rp.astype(np.int32)), L.iptr(col.astype(np.int32)),
                                     L.dptr(val.astype(np.float64))))
    assert lib.lsg_solve(ctx.h, L.dptr(b), L.dptr(x), ctypes.byref(st)) == L.LSG_ERR_STATE
    # projection entry points without geometry
    out = np.empty(n)
    assert lib.lsg_projection_rhs(ctx.h, L.dptr(out), L.dptr(out), L.dptr(out), L.dptr(out),
                                  L.dptr(out)) == L.LSG_ERR_STATE
    ctx.close()
    # the solver mirror raises on the same errors
    s = S.MGFGMRES()
    with pytest.raises(L.LsgError) as e:
        s.set(_csr(g), task=S.Task(), setup=False)
        s.solve(g["b"], np.zeros(n))
    assert e.value.code == L.LSG_ERR_STATE
    s.close()


def test_operator_outside_the_stencil_is_rejected():
    from lsstag_b200 import _lib as L
    from lsstag_b200 import solver as S
    g = load_golden("sphere16")
    rp, col, val = (np.array(g[k]) for k in ("A_rowptr", "A_col", "A_val"))
    dims = tuple(int(v) for v in g["dims"])
    N = dims[0]
    # row 200's first entry pointed two cells away (not a face neighbour)
    r = 200
    col[rp[r]] = r + 2 if col[rp[r]] != r + 2 else r - 2
    s = S.MGFGMRES()
    with pytest.raises(L.LsgError) as e:
        s.set((rp, col, val, dims))
    assert e.value.code == L.LSG_ERR_PATTERN
    assert N > 2
    s.close()


def test_bounded_wait_runs_out_and_is_reported():
    """The one-launch ILU(0) sweep waits at a grid barrier between
    hyperplanes for one second at most.  The self-test entry point runs it
    with one CTA leaving before its first arrival: the others' wait runs
    out, the kernel ends with its flag set, the call returns LSG_ERR_CUDA
    with the reason, and the same context then solves normally."""
    import time

    from lsstag_b200 import _lib as L
    from lsstag_b200 import cases
    from lsstag_b200 import solver as S
    P, dims, pins, b = cases.load(128)
    s = S.ILUFGMRES()
    s.set_planes(P, dims, S.Task(eps=1e-8 * float(np.linalg.norm(b))))
    t0 = time.perf_counter()
    rc = s.ctx.lib.lsg_selftest_wait_limit(s.ctx.h)
    dt = time.perf_counter() - t0
    msg = s.ctx.lib.lsg_last_error(s.ctx.h).decode()
    print(f"wait-limit self-test: rc {rc} after {dt:.2f} s: {msg}")
    assert rc == L.LSG_ERR_CUDA and "barrier" in msg
    assert 0.5 < dt < 60
    # the context then solves as a fresh one does, to the bit
    x = np.zeros(b.size)
    its = s.solve(b, x)
    s.close()
    f = S.ILUFGMRES()
    f.set_planes(P, dims, S.Task(eps=1e-8 * float(np.linalg.norm(b))))
    xf = np.zeros(b.size)
    itf = f.solve(b, xf)
    f.close()
    assert its == itf and np.array_equal(x, xf) and np.all(np.isfinite(x))

