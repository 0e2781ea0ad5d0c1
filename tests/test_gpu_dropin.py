"""The drop-in itself: the reference's own time step and pressure equation
(TimeSteppingMethodInterface::step order, PoissonDiscreteEquation::solve,
time_stepping_method_interface.h:180-214, poisson_discrete_equation.h:167-209)
compiled with -DLS_STAG_USE_B200, so that the equation's solver member is
include/lsstag_b200_adapter.hpp's B200MGFGMRES calling the library through
the C ABI (oracle/_ref/ref_harness_b200, built by oracle/build_ref.sh).  Its
results are compared with the stock reference build's on the same cases:
iteration counts within +-1, states within 1e-10 relative L2."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _binaries():
    import ref_runner as rr
    if not (rr.available(rr.REF_BIN) and rr.available(rr.DROPIN_BIN)):
        pytest.fail("oracle/_ref/ref_harness and ref_harness_b200 must be built (oracle/build_ref.sh)")
    return rr


def test_reference_time_steps_with_b200_pressure_solver():
    """Three whole time steps of the 16^3 sphere flow, every equation solved
    to an absolute 1e-11: the reference's momentum solvers, its pressure
    equation with the B200 solver swapped in."""
    rr = _binaries()
    h = 1.0 / 16
    case = rr.Case(16, 16, 16, h, h, h, spheres=[(0.5 + 0.3 * h, 0.5 + 0.2 * h, 0.5 + 0.1 * h, 0.18)])
    kw = dict(threads=1, flow_steps=3, task_eps=1e-11, restart=30, dump_geometry=0)
    ref = rr.run(case, **kw)
    drop = rr.run(case, binary=rr.DROPIN_BIN, **kw)
    for s in (1, 2, 3):
        its_r, its_d = ref[f"its_{s}"], drop[f"its_{s}"]
        assert all(abs(int(a) - int(b)) <= 1 for a, b in zip(its_d, its_r)), (s, its_d, its_r)
        for k in ("u", "v", "w", "p", "phi"):
            e = _rel(drop[f"{k}_{s}"], ref[f"{k}_{s}"])
            assert e <= 1e-10, (s, k, e)


def test_reference_pressure_solve_with_b200_solver():
    """The pressure equation's own solve (the harness's MG-FGMRES mode runs
    pEq->solver) on the four-sphere 24^3 case to a 1e-10 relative residual."""
    rr = _binaries()
    from lsstag_b200 import synth
    h = 1.0 / 24
    case = rr.Case(24, 24, 24, h, h, h, spheres=synth.four_spheres(3, rmin=0.05, rmax=0.1, cmin=0.4, cmax=0.6))
    g = rr.run(case, threads=1, fgmres=0, dump_geometry=1)
    rp, col, val, _ = rr.csr(g, "A")
    mask = synth.connected_fluid(rp, col, val, g["pins"])
    b = synth.poisson_rhs(7, g["celltype"], g["pins"], mask)
    kw = dict(threads=1, fgmres=1, bicgstab=0, dump_geometry=0, restart=30, rel_tol=1e-10, max_it=200)
    ref = rr.run(case, b, **kw)
    drop = rr.run(case, b, binary=rr.DROPIN_BIN, **kw)
    assert abs(int(drop["fgmres_it"][0]) - int(ref["fgmres_it"][0])) <= 1
    assert _rel(drop["fgmres_x"], ref["fgmres_x"]) <= 1e-10
