"""The native flow time step (lsg_flow_create / lsg_flow_step,
csrc/lsg_flow.cu: C++ drives the step, the three momentum solves run on
library threads) against the reference's own steps on the 16^3 sphere flow
(iterations within 1, fields within 1e-9 relative L2, as
tests/test_gpu_flow.py) and against the Python-driven device stepper
(FlowStepperDevice) bit for bit: the same entry points run on the same
inputs in the same order; the driver only changes who issues them.  Also on
the 128x64x64 flow set up from the sphere on the device, with the pressure
solved relative to ||b||; and the stepper's errors."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def _par(g):
    nu, coef, coef2, integr, dt, eps, vbase, maxit = (float(v) for v in g["nu_coef_coef2_integr_dt_eps_vbase_maxit"])
    return dict(nu=nu, coef=coef, coef2=coef2, coef_integr=integr, eps=eps, vbase=vbase, max_it=int(maxit),
                restart_mom=int(g["restart_mom_p"][0]), restart_p=int(g["restart_mom_p"][1]))


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def test_native_steps_match_reference_and_device_stepper():
    from lsstag_b200.flow import FlowStepperDevice, FlowStepperNative
    g = load_golden("flow16_steps")
    par = _par(g)
    fn = FlowStepperNative(g, g["dims"], par, g["u_0"], g["v_0"], g["w_0"], g["p_0"])
    fd = FlowStepperDevice(g, g["dims"], par, g["u_0"], g["v_0"], g["w_0"], g["p_0"])
    for s in (1, 2, 3):
        its = fn.step()
        its_d = fd.step()
        assert its == list(its_d)
        for a, b in zip(its, g[f"its_{s}"]):
            assert abs(int(a) - int(b)) <= 1, (s, its, g[f"its_{s}"])
        (u, v, w), p = fn.state()
        (ud, vd, wd), pd = fd.state()
        for name, mine, dev in zip("uvw", (u, v, w), (ud, vd, wd)):
            assert _rel(mine, g[f"{name}_{s}"]) <= 1e-9, (s, name)
            assert mine.tobytes() == dev.tobytes(), (s, name)
        assert _rel(p, g[f"p_{s}"]) <= 1e-9
        assert p.tobytes() == pd.tobytes()
    fn.close()
    fd.close()


def test_native_steps_128_relative_pressure_tolerance():
    """Two steps of the 128x64x64 flow (mesh built on the device from the
    sphere), pressure to 1e-9 relative to ||b|| with the FP32 cycle: native
    and Python-driven steppers agree bit for bit."""
    from lsstag_b200 import cases
    from lsstag_b200.flow import FlowStepperDevice, FlowStepperNative
    h = 1.0 / 16
    g, dims, par, st = cases.flow_case_on_device((128, 64, 64), (h, h, h),
                                                 spheres=[(2.0, 2.0 + 0.5 * h, 2.0 + 0.5 * h, 0.5)])
    kw = dict(pressure_mg_fp32=True, p_rel_tol=1e-9)
    fn = FlowStepperNative(g, dims, par, *st, **kw)
    fd = FlowStepperDevice(g, dims, par, *st, **kw)
    for _ in range(2):
        assert fn.step() == list(fd.step())
    (u, v, w), p = fn.state()
    (ud, vd, wd), pd = fd.state()
    for a, b in zip((u, v, w, p), (ud, vd, wd, pd)):
        assert a.tobytes() == b.tobytes()
    fn.close()
    fd.close()


def test_native_stepper_errors():
    import ctypes

    from lsstag_b200 import _lib as L
    lib = L.load()
    h = ctypes.c_void_p()
    d = L.FlowDesc()                                       # no contexts, no arrays
    d.N, d.M, d.K = 8, 8, 8
    assert lib.lsg_flow_create(ctypes.byref(d), ctypes.byref(h)) == L.LSG_ERR_ARG
    assert not h.value
    from lsstag_b200.flow import FlowStepperNative
    g = load_golden("flow16_steps")
    fn = FlowStepperNative(g, g["dims"], _par(g), g["u_0"], g["v_0"], g["w_0"], g["p_0"])
    # a second stepper on the same contexts: a step before its state is set
    h2 = ctypes.c_void_p()
    assert lib.lsg_flow_create(ctypes.byref(fn.desc), ctypes.byref(h2)) == L.LSG_OK
    its = (ctypes.c_int * 4)()
    assert lib.lsg_flow_step(h2, its) == L.LSG_ERR_STATE
    assert b"lsg_flow_set_state" in lib.lsg_flow_last_error(h2)
    lib.lsg_flow_destroy(h2)
    # a negative relative tolerance is refused
    d3 = L.FlowDesc.from_buffer_copy(fn.desc)
    d3.p_rel_tol = -1.0
    assert lib.lsg_flow_create(ctypes.byref(d3), ctypes.byref(h2)) == L.LSG_ERR_ARG
    fn.close()
