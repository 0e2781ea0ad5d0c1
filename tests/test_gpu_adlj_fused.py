"""The fused ADLJ direction step (LSG_ADLJ_FUSED, the default of the FP32
cycle under LSG_ADLJ_AUTO: one kernel
per direction forms the residual b - A ch inside its line solve and writes
ch + omega T_d^{-1} (b - A ch)) against the reference's schedule
(LSG_ADLJ_REFERENCE: r -= A c, c = omega T_d^{-1} r, ch += c as separate
kernels, smoother_adlj_interface.h:66-77).  The two are equal in exact
arithmetic, so one V-cycle agrees to rounding (a wrong coefficient, stride or
buffer would show as an O(1) difference) and whole solves take the same
iteration counts.  The fused kernels run on the levels with the 7-point
stencil whose x-lines split into 8-cell segments over a power-of-two number
of lanes (sphere16, the 128^3 four-sphere case); the coarse Galerkin levels
keep the separate kernels."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def _csr(g):
    return (g["A_rowptr"], g["A_col"], g["A_val"], tuple(int(v) for v in g["dims"]))


@pytest.mark.parametrize("case", ["sphere16", "spheres4_24"])
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_vcycle_matches_reference_schedule_sphere16(prec, case):
    """sphere16 splits its x-lines into 8-cell segments (2 lanes), spheres4_24
    into 12-cell ones (2 lanes)."""
    from lsstag_b200 import _lib as L
    from lsstag_b200 import solver as S
    g = load_golden(case)
    p = L.FP64 if prec == "fp64" else L.FP32
    out, its = [], []
    for sched in (L.ADLJ_FUSED, L.ADLJ_REFERENCE):
        s = S.MGFGMRES(mg_precision=p, adlj_schedule=sched)
        s.set(_csr(g), task=S.Task(eps=float(g["eps"][0])))
        out.append(s.precondition(g["b"]))
        x = np.zeros(g["b"].size)
        its.append(s.solve(g["b"], x))
        s.close()
    rel = np.linalg.norm(out[0] - out[1]) / np.linalg.norm(out[1])
    print(f"{case} {prec}: one V-cycle, fused vs reference schedule, relative {rel:.2e}; iterations {its}")
    assert rel <= (1e-12 if prec == "fp64" else 1e-5)
    assert abs(its[0] - its[1]) <= 1
    assert its[1] == int(g["fgmres_it"][0]) or prec == "fp32"


@pytest.fixture(scope="module")
def case128():
    from lsstag_b200 import cases
    return cases.load(128)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_vcycle_and_solve_128(case128, prec):
    from lsstag_b200 import _lib as L
    from lsstag_b200 import solver as S
    P, dims, pins, b = case128
    p = L.FP64 if prec == "fp64" else L.FP32
    tol = 1e-10 * float(np.linalg.norm(b))
    out, its, xs = [], [], []
    for sched in (L.ADLJ_FUSED, L.ADLJ_REFERENCE):
        s = S.MGFGMRES(mg_precision=p, adlj_schedule=sched)
        s.set_planes(P, dims, S.Task(eps=tol, FGMRES_RESTART_NUM=30))
        out.append(s.precondition(b))
        x = np.zeros(b.size)
        its.append(s.solve(b, x))
        assert s.status == L.LSG_OK
        assert s.stats.true_residual <= 1.5 * tol
        xs.append(x)
        s.close()
    rel = np.linalg.norm(out[0] - out[1]) / np.linalg.norm(out[1])
    dx = np.linalg.norm(xs[0] - xs[1]) / np.linalg.norm(xs[1])
    print(f"128^3 {prec}: V-cycle relative {rel:.2e}; iterations {its}; solutions relative {dx:.2e}")
    assert rel <= (1e-12 if prec == "fp64" else 1e-5)
    assert abs(its[0] - its[1]) <= 1
    # both solutions meet the 1e-10 relative residual; the operator's
    # conditioning lets such solutions differ by a few 1e-8 (the FP32 and FP64
    # cycles' solutions of this system differ by 5e-8)
    assert dx <= 1e-6


def _long_case(dims, seed=3):
    """(planes, rhs) of the four seeded spheres in the unit cube on an
    N x M x K grid, operator built on the GPU (as cases.build_on_device)."""
    from lsstag_b200 import cases, mesh as MS, solver as S, synth
    N, M, K = dims
    h = (1.0 / N, 1.0 / M, 1.0 / K)
    sph = synth.four_spheres(seed)
    pins = np.array([N - 1, N * M - 1], dtype=np.int64)
    s = S.MGFGMRES()
    try:
        s.build_mesh(dims, h, MS.flow_block(dims, h, sph), bodies=MS.bodies_array(sph))
        s.set_from_mesh(pins, setup=False)
        P = s.planes()
        solid = s.mesh_get("celltype") == 0
    finally:
        s.close()
    mask = cases.fluid_mask_from_planes(P, dims, pins)
    return P, synth.poisson_rhs(seed, np.where(solid, 0, 1), pins, mask)


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
@pytest.mark.parametrize("dims", [(512, 16, 16), (384, 16, 16), (16, 384, 16), (16, 16, 384)])
def test_long_lines_fused_match_reference_schedule(dims, prec):
    """Lines longer than 256 cells in the FP32 cycle: x-lines of 512 in
    16-cell segments and of 384 in 12-cell ones (32 lanes), y-lines of 384 in
    8-cell segments (48 per line), z-lines of 384 in 12-cell ones; one
    V-cycle against the reference's schedule to rounding (FP32 cycle; the
    FP64 cycle with the fused schedule asked for explicitly, which fuses the
    x-lines of 512 and 384 and keeps the reference's schedule where 8-cell
    FP64 segments would exceed 256 threads: 0 difference there), the same
    iterations to the same 1e-10 relative residual."""
    from lsstag_b200 import _lib as L
    from lsstag_b200 import solver as S
    P, b = _long_case(dims)
    tol = 1e-10 * float(np.linalg.norm(b))
    out, its = [], []
    for sched in (L.ADLJ_FUSED, L.ADLJ_REFERENCE):
        s = S.MGFGMRES(mg_precision=L.FP32 if prec == "fp32" else L.FP64, adlj_schedule=sched)
        s.set_planes(P, dims, S.Task(eps=tol, FGMRES_RESTART_NUM=30, MAX_ITER=200))
        out.append(s.precondition(b))
        x = np.zeros(b.size)
        its.append(s.solve(b, x))
        assert s.status == L.LSG_OK
        assert s.stats.true_residual <= 1.5 * tol
        s.close()
    rel = np.linalg.norm(out[0] - out[1]) / np.linalg.norm(out[1])
    print(f"{dims} {prec}: one V-cycle, fused vs reference schedule, relative {rel:.2e}; iterations {its}")
    assert rel <= (1e-5 if prec == "fp32" else 1e-12)
    assert abs(its[0] - its[1]) <= 1


def test_fused_steps_profiled_128(case128):
    """Kernel ids 9/10/11 (the fused x/y/z steps on the finest level) run
    and report their algorithmic bytes (4w + 4 per cell); the reference
    schedule's context refuses them."""
    import ctypes
    from lsstag_b200 import _lib as L
    from lsstag_b200 import solver as S
    P, dims, pins, b = case128
    n = int(np.prod(dims))
    s = S.MGFGMRES(mg_precision=L.FP32)
    s.set_planes(P, dims, S.Task(eps=1e-10 * float(np.linalg.norm(b))))
    for k in (9, 10, 11):
        ms, by = ctypes.c_double(), ctypes.c_double()
        s.ctx.check(s.ctx.lib.lsg_profile_kernel(s.ctx.h, k, 5, ctypes.byref(ms), ctypes.byref(by)))
        assert ms.value > 0 and by.value == 20.0 * n
        print(f"fused step {k}: {ms.value * 1e3:.1f} us, {by.value / ms.value / 1e6:.0f} GB/s")
    s.close()
    r = S.MGFGMRES(mg_precision=L.FP32, adlj_schedule=L.ADLJ_REFERENCE)
    r.set_planes(P, dims, S.Task(eps=1e-10 * float(np.linalg.norm(b))))
    ms, by = ctypes.c_double(), ctypes.c_double()
    assert r.ctx.lib.lsg_profile_kernel(r.ctx.h, 9, 1, ctypes.byref(ms), ctypes.byref(by)) == L.LSG_ERR_STATE
    r.close()
