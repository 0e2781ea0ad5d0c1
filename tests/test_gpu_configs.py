"""Parity at the measured configurations' own sizes, against the reference
run on the same system in the same process tree (oracle/_ref/ref_harness,
the reference's own MGFGMRES / time step compiled from its sources).

* 128^3 four-sphere Poisson system (seed 3), MG-FGMRES(30) to a 1e-10
  relative residual (the reference's absolute stop at 1e-10 ||b||,
  fgmres_interface.h:78-142): FP64 iterations within +-1 and solution
  within 1e-10 relative L2; FP32 multigrid inside FP64 FGMRES within the
  mixed-precision tolerance stated below.
* The 128x64x64 sphere flow: ten reference time steps
  (TimeSteppingMethodInterface::step, time_stepping_method_interface.h:180-214)
  against ten GPU steps from the same initial state.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def c1_128():
    import ref_runner as rr
    from lsstag_b200 import cases
    if not rr.available():
        pytest.fail("oracle/_ref/ref_harness is not built (run __graft_entry__.build() where the reference is)")
    P, dims, pins, b = cases.load(128)
    threads = os.cpu_count() or 1
    ref = rr.run_planes(P, dims, b, threads=threads, fgmres=1, bicgstab=0, restart=30, rel_tol=1e-10, max_it=200)
    return P, dims, b, ref


def test_c1_128_fp64_matches_reference(c1_128):
    from lsstag_b200 import solver as S
    P, dims, b, ref = c1_128
    eps = float(ref["eps"][0])
    s = S.MGFGMRES()
    s.set_planes(P, dims, task=S.Task(eps=eps, FGMRES_RESTART_NUM=30, MAX_ITER=200))
    x = np.zeros(b.size)
    it = s.solve(b, x)
    it_ref = int(ref["fgmres_it"][0])
    err = _rel(x, ref["fgmres_x"])
    print(f"128^3 FP64: iterations {it} (reference {it_ref}), rel L2 to the reference {err:.3e}")
    assert abs(it - it_ref) <= 1
    assert err <= 1e-10
    assert s.stats.true_residual <= eps * 1.0000001
    s.close()


def test_c1_128_fp32_mg_matches_reference(c1_128):
    """FP32 multigrid inside FP64 FGMRES with iterative refinement: the FP64
    true residual meets 1e-10 ||b||, and the solution lies within 1e-6
    (relative L2) of the reference's FP64 one.  Both solutions stop at a
    relative residual of 1e-10 along different Krylov paths, so they may
    differ by up to 1e-10 times the operator's condition number (about 1e4
    relative to the solution here); the measured gap is far below."""
    from lsstag_b200 import _lib as L
    from lsstag_b200 import solver as S
    P, dims, b, ref = c1_128
    eps = float(ref["eps"][0])
    s = S.MGFGMRES(mg_precision=L.FP32)
    s.set_planes(P, dims, task=S.Task(eps=eps, FGMRES_RESTART_NUM=30, MAX_ITER=200))
    x = np.zeros(b.size)
    it = s.solve(b, x)
    err = _rel(x, ref["fgmres_x"])
    print(f"128^3 FP32-MG: iterations {it} (reference FP64 {int(ref['fgmres_it'][0])}), "
          f"rel L2 to the reference {err:.3e}")
    assert s.stats.true_residual <= eps * 1.0000001
    assert abs(it - int(ref["fgmres_it"][0])) <= 2
    assert err <= 1e-6
    s.close()


def test_c0_flow_ten_steps_match_reference():
    """Ten time steps of the flow past a sphere at 128x64x64 (domain
    [0,8]x[0,4]x[0,4], D = 1, Re 100, dt 0.01, FGMRES(30) pressure,
    ILU(0)-FGMRES(13) momentum, every equation to an absolute residual of
    1e-9) from the reference's initial state, on the reference's own mesh
    build of this run.

    The bar is the reference against itself.  Its pressure solve on this
    flow sits near the attainable accuracy of the operator, so the
    reference's own result moves with its OpenMP thread count: at 1e-9,
    1 and 8 threads give the same iteration counts but pressures 5e-8 apart
    after two steps; at 1e-10 and 1e-11 even the counts differ (11 against
    20, 21 against 23).  So the reference runs here with 1, 2, 4 and all host
    threads (how far the runs spread depends on the host's thread count:
    1 against 16 threads gave 1.0e-8 in p after one step, while the GPU's p
    lies 4.5e-8 from the 1-thread run); the GPU's iteration counts must lie
    within their band +-1 and each field within max(4 x their spread so far,
    1e-10) of the 1-thread run, the spread being the largest distance of a
    reference run from the 1-thread one."""
    import ref_runner as rr
    from lsstag_b200.flow import FlowStepperDevice
    if not rr.available():
        pytest.fail("oracle/_ref/ref_harness is not built")
    h = 1.0 / 16
    case = rr.Case(128, 64, 64, h, h, h, spheres=[(2.0, 2.0 + 0.5 * h, 2.0 + 0.5 * h, 0.5)])
    steps = 10
    kw = dict(flow_steps=steps, restart=30, dump_geometry=0, task_eps=1e-9, timeout=3000)
    r = rr.run(case, threads=1, **kw)
    nmax = os.cpu_count() or 1
    runs = [rr.run(case, threads=t, **kw) for t in sorted({min(2, nmax), min(4, nmax), nmax}) if t > 1]
    rn = runs[-1]
    dims = tuple(int(v) for v in r["dims"])
    nu, coef, coef2, integr, dt, eps, vbase, maxit = (float(v) for v in r["nu_coef_coef2_integr_dt_eps_vbase_maxit"])
    assert eps == 1e-9
    par = dict(nu=nu, coef=coef, coef2=coef2, coef_integr=integr, eps=eps, vbase=vbase, max_it=int(maxit),
               restart_mom=int(r["restart_mom_p"][0]), restart_p=int(r["restart_mom_p"][1]))
    fs = FlowStepperDevice(r, dims, par, r["u_0"], r["v_0"], r["w_0"], r["p_0"])
    spread = np.zeros(4)
    for s in range(1, steps + 1):
        its = fs.step()
        i1 = [int(v) for v in r[f"its_{s}"]]
        i_n = [int(v) for v in rn[f"its_{s}"]]
        bands = [[int(v) for v in q[f"its_{s}"]] for q in runs]
        (u, v, w), p = fs.state()
        fields = ("u", "v", "w", "p")
        errs = [_rel(a, r[f"{k}_{s}"]) for a, k in zip((u, v, w, p), fields)]
        for q in runs:
            spread = np.maximum(spread, [_rel(q[f"{k}_{s}"], r[f"{k}_{s}"]) for k in fields])
        print(f"C0 step {s}: iterations {its} (reference 1 thread {i1}, all threads {i_n}), "
              f"rel L2 u v w p {['%.2e' % e for e in errs]}, reference spread {['%.2e' % e for e in spread]}")
        for e_, a in enumerate(its):
            band = [i1[e_]] + [q[e_] for q in bands]
            assert min(band) - 1 <= int(a) <= max(band) + 1, (s, its, i1, bands)
        for e, sp in zip(errs, spread):
            assert e <= max(4.0 * sp, 1e-10), (s, errs, spread.tolist())
    fs.close()
