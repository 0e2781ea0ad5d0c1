"""Whole time steps of the flow past a sphere with every operator on the GPU
(lsstag_b200.flow.FlowStepper: momentum operators and source terms from the
geometry, convective terms matrix-free, ILU(0)-FGMRES momentum solves,
MG-FGMRES pressure solve, projection) against the reference's own time steps
(TimeSteppingMethodInterface::step) from the same initial state: iteration
counts within 1 and velocities / pressure within 1e-9 relative L2 after each
of three steps (both sides solve to an absolute residual of 1e-11)."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def _stepper():
    from lsstag_b200.flow import FlowStepper
    g = load_golden("flow16_steps")
    nu, coef, coef2, integr, dt, eps, vbase, maxit = (float(v) for v in g["nu_coef_coef2_integr_dt_eps_vbase_maxit"])
    par = dict(nu=nu, coef=coef, coef2=coef2, coef_integr=integr, eps=eps, vbase=vbase, max_it=int(maxit),
               restart_mom=int(g["restart_mom_p"][0]), restart_p=int(g["restart_mom_p"][1]))
    fs = FlowStepper(g, g["dims"], par, g["u_0"], g["v_0"], g["w_0"], g["p_0"])
    return g, fs


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def test_flow_steps_match_reference():
    g, fs = _stepper()
    for s in (1, 2, 3):
        its = fs.step()
        ref_its = g[f"its_{s}"]
        for a, b in zip(its, ref_its):
            assert abs(int(a) - int(b)) <= 1, (s, its, ref_its)
        for k, (mine, ref) in enumerate(zip(fs.predictions, (g[f"us_{s}"], g[f"vs_{s}"], g[f"ws_{s}"]))):
            assert _rel(mine, ref) <= 1e-9, (s, "prediction", k, _rel(mine, ref))
        assert _rel(fs.phi, g[f"phi_{s}"]) <= 1e-9, (s, "phi", _rel(fs.phi, g[f"phi_{s}"]))
        for name, mine in zip("uvw", fs.u):
            assert _rel(mine, g[f"{name}_{s}"]) <= 1e-9, (s, name, _rel(mine, g[f"{name}_{s}"]))
        assert _rel(fs.p, g[f"p_{s}"]) <= 1e-9, (s, "p", _rel(fs.p, g[f"p_{s}"]))
    fs.close()


def test_flow_steps_device_resident_match_reference():
    """The device-resident stepper (state in device memory, *_device entry
    points) gives the same steps."""
    from lsstag_b200.flow import FlowStepperDevice
    g = load_golden("flow16_steps")
    nu, coef, coef2, integr, dt, eps, vbase, maxit = (float(v) for v in g["nu_coef_coef2_integr_dt_eps_vbase_maxit"])
    par = dict(nu=nu, coef=coef, coef2=coef2, coef_integr=integr, eps=eps, vbase=vbase, max_it=int(maxit),
               restart_mom=int(g["restart_mom_p"][0]), restart_p=int(g["restart_mom_p"][1]))
    fs = FlowStepperDevice(g, g["dims"], par, g["u_0"], g["v_0"], g["w_0"], g["p_0"])
    for s in (1, 2, 3):
        its = fs.step()
        for a, b in zip(its, g[f"its_{s}"]):
            assert abs(int(a) - int(b)) <= 1, (s, its, g[f"its_{s}"])
        (u, v, w), p = fs.state()
        for name, mine in zip("uvw", (u, v, w)):
            assert _rel(mine, g[f"{name}_{s}"]) <= 1e-9, (s, name)
        assert _rel(p, g[f"p_{s}"]) <= 1e-9, (s, "p")
    fs.close()
