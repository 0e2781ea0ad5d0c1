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
    ILU(0)-FGMRES(13) momentum) from the reference's initial state, every
    equation solved to an absolute residual of 1e-11 on both sides: iteration
    counts within +-1 and u, v, w, p within 1e-10 relative L2 after every
    step.  The mesh arrays the GPU steps read are the reference's own mesh
    build of this run."""
    import ref_runner as rr
    from lsstag_b200.flow import FlowStepperDevice
    if not rr.available():
        pytest.fail("oracle/_ref/ref_harness is not built")
    h = 1.0 / 16
    case = rr.Case(128, 64, 64, h, h, h, spheres=[(2.0, 2.0 + 0.5 * h, 2.0 + 0.5 * h, 0.5)])
    steps = 10
    r = rr.run(case, threads=os.cpu_count() or 1, flow_steps=steps, restart=30, dump_geometry=0,
               task_eps=1e-11, timeout=3000)
    dims = tuple(int(v) for v in r["dims"])
    nu, coef, coef2, integr, dt, eps, vbase, maxit = (float(v) for v in r["nu_coef_coef2_integr_dt_eps_vbase_maxit"])
    assert eps == 1e-11
    par = dict(nu=nu, coef=coef, coef2=coef2, coef_integr=integr, eps=eps, vbase=vbase, max_it=int(maxit),
               restart_mom=int(r["restart_mom_p"][0]), restart_p=int(r["restart_mom_p"][1]))
    fs = FlowStepperDevice(r, dims, par, r["u_0"], r["v_0"], r["w_0"], r["p_0"])
    worst = 0.0
    for s in range(1, steps + 1):
        its = fs.step()
        ref_its = [int(v) for v in r[f"its_{s}"]]
        (u, v, w), p = fs.state()
        errs = [_rel(u, r[f"u_{s}"]), _rel(v, r[f"v_{s}"]), _rel(w, r[f"w_{s}"]), _rel(p, r[f"p_{s}"])]
        worst = max(worst, max(errs))
        print(f"C0 step {s}: iterations {its} (reference {ref_its}), rel L2 u v w p {errs}")
        assert all(abs(int(a) - b) <= 1 for a, b in zip(its, ref_its)), (s, its, ref_its)
        assert max(errs) <= 1e-10, (s, errs)
    fs.close()
    print("C0 worst rel L2 over 10 steps:", worst)
