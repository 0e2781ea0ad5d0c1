"""Cut-cell loads on the GPU through the C ABI (lsg_loads_*), against the
reference's own LoadsCalculator outputs: every cut-cell type on seeded
arrays, and calculate() on a sphere's cut cells.  Per-cell forces are
bitwise equal; sums and moments agree to 1e-13 relative (summation order);
the adjoint agrees with the CPU restatement and with directional
differences of the forward loads."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def _probe_calc(g, nucell=None):
    from lsstag_b200.loads import LoadsCalculator
    lc = LoadsCalculator()
    lc.set(g["dims"], g["cells"], g["type"], g["theta"], g["delta"], g["invv"], g["dmax"], g["dne"], g["dtn"],
           g["nodes"], g["center"], 2.0, 0.01)
    lc.calculate(g["ux"], g["uy"], g["uz"], g["p"], g["vib"], g["vibyx"], g["vibzy"], float(g["nu"]),
                 nu_cell=nucell)
    return lc


@pytest.mark.parametrize("per_cell_nu", [False, True])
def test_loads_every_cell_type_bitwise(per_cell_nu):
    g = load_golden("loads_probe")
    sfx = "_nucell" if per_cell_nu else ""
    lc = _probe_calc(g, g["nucell"] if per_cell_nu else None)
    for got, k in zip((lc.ForceX, lc.ForceY, lc.ForceZ), ("fx", "fy", "fz")):
        assert np.array_equal(got, g[k + sfx]), k
    for c, k in enumerate(("fx", "fy", "fz")):
        ref = g[k + sfx]
        assert abs((lc.F_aer_x, lc.F_aer_y, lc.F_aer_z)[c] - ref.sum()) <= 1e-13 * np.abs(ref).sum()
    for c, k in enumerate(("mz", "mx", "my")):
        ref = g[k + sfx]
        assert abs(lc.moment_raw[c] - ref.sum()) <= 1e-13 * np.abs(ref).sum()
    lc.close()


def test_loads_calculate_on_sphere():
    from lsstag_b200.loads import LoadsCalculator
    import lsg_oracle as O
    r = load_golden("loads_sphere16")
    nu, fcoef, dt = (float(v) for v in r["nu_fcoef_dt"])
    lc = LoadsCalculator()
    lc.set(r["dims"], r["cells"], r["celltype"], r["theta"], r["delta"], r["inv_vof"], r["dmax"], r["dne"],
           r["dtn"], r["nodes"], r["center"], fcoef, dt)
    lc.calculate(r["ux"], r["uy"], r["uz"], r["p"], r["vib"], r["vibyx"], r["vibzy"], nu)
    for got, k in zip((lc.ForceX, lc.ForceY, lc.ForceZ), ("fx", "fy", "fz")):
        assert np.array_equal(got, r[k]), k
    sums = r["sums"]
    got = [lc.F_aer_x, lc.F_aer_y, lc.F_aer_z, lc.C_d, lc.C_y, lc.C_z, lc.moment_aer, lc.moment_x_aer,
           lc.moment_y_aer]
    m = O.loads_moments(r["cells"], r["nodes"], r["center"], r["fx"], r["fy"], r["fz"])
    fs = [np.abs(r[k]).sum() for k in ("fx", "fy", "fz")]
    scale = fs + [v * fcoef for v in fs] + [np.abs(mm).sum() for mm in m]
    for i in range(9):
        assert abs(got[i] - sums[i]) <= 1e-13 * scale[i], i
    # the moment filters advance one step per call, like the reference's
    flt = [O.LoadsFilter(dt) for _ in range(3)]
    lc.reset_filter(dt)
    for rep in range(4):
        sc = 1.0 + 0.25 * rep
        lc.calculate(r["ux"] * sc, r["uy"] * sc, r["uz"] * sc, r["p"] * sc, r["vib"] * sc, r["vibyx"] * sc,
                     r["vibzy"] * sc, nu)
        if rep == 0:
            expect = [f.step(mm.sum()) for f, mm in zip(flt, m)]
        else:
            f2 = O.loads_forces(*(int(v) for v in r["dims"]), r["cells"], r["celltype"], r["theta"], r["delta"],
                                r["inv_vof"], r["dmax"], r["dne"], r["dtn"], r["vib"] * sc, r["vibyx"] * sc,
                                r["vibzy"] * sc, r["ux"] * sc, r["uy"] * sc, r["uz"] * sc, r["p"] * sc, nu)
            m2 = O.loads_moments(r["cells"], r["nodes"], r["center"], *f2)
            expect = [f.step(mm.sum()) for f, mm in zip(flt, m2)]
        for c, e in enumerate(expect):
            got_m = (lc.moment_aer, lc.moment_x_aer, lc.moment_y_aer)[c]
            assert abs(got_m - e) <= 1e-12 * max(1.0, abs(e)), (rep, c)
    lc.close()


def test_loads_device_entry_matches_host_entry():
    import torch
    g = load_golden("loads_sphere16")
    from lsstag_b200.loads import LoadsCalculator
    nu, fcoef, dt = (float(v) for v in g["nu_fcoef_dt"])
    lcs = []
    for _ in range(2):
        lc = LoadsCalculator()
        lc.set(g["dims"], g["cells"], g["celltype"], g["theta"], g["delta"], g["inv_vof"], g["dmax"], g["dne"],
               g["dtn"], g["nodes"], g["center"], fcoef, dt)
        lcs.append(lc)
    lcs[0].calculate(g["ux"], g["uy"], g["uz"], g["p"], g["vib"], g["vibyx"], g["vibzy"], nu)
    dev = {k: torch.from_numpy(np.ascontiguousarray(g[k])).cuda() for k in
           ("ux", "uy", "uz", "p", "vib", "vibyx", "vibzy")}
    forces = torch.empty(3 * g["cells"].size, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    lcs[1].calculate_device(*(dev[k].data_ptr() for k in ("ux", "uy", "uz", "p", "vib", "vibyx", "vibzy")), nu,
                            forces=forces.data_ptr())
    f = forces.cpu().numpy()
    c = g["cells"].size
    assert np.array_equal(f[:c], lcs[0].ForceX) and np.array_equal(f[2 * c:], lcs[0].ForceZ)
    assert lcs[1].C_d == lcs[0].C_d and lcs[1].moment_aer == lcs[0].moment_aer
    for lc in lcs:
        lc.close()


@pytest.mark.parametrize("per_cell_nu", [False, True])
def test_loads_adjoint(per_cell_nu):
    """Gradient of w . (F_aer_x, F_aer_y, F_aer_z) against the CPU
    restatement (1e-12) and against directional differences of the GPU
    forward loads (the loads are affine in the fields)."""
    import lsg_oracle as O
    g = load_golden("loads_probe")
    N, M, K = (int(v) for v in g["dims"])
    nucell = g["nucell"] if per_cell_nu else None
    w = np.array([1.0, -0.5, 0.25])
    lc = _probe_calc(g, nucell)
    grads = lc.adjoint(w, float(g["nu"]), nu_cell=nucell)
    ref = O.loads_adjoint(N, M, K, g["cells"], g["type"], g["theta"], g["delta"], g["invv"], g["dmax"], g["dne"],
                          g["dtn"], w, float(g["nu"]), nu_cell=nucell)
    for a, b in zip(grads, ref):
        assert np.linalg.norm(a - b) <= 1e-12 * np.linalg.norm(b)
    J0 = w @ np.array([lc.F_aer_x, lc.F_aer_y, lc.F_aer_z])
    rng = np.random.default_rng(9)
    d = [rng.normal(size=a.size) for a in grads]
    lc.calculate(g["ux"] + d[0], g["uy"] + d[1], g["uz"] + d[2], g["p"] + d[3], g["vib"], g["vibyx"],
                 g["vibzy"], float(g["nu"]), nu_cell=nucell)
    J1 = w @ np.array([lc.F_aer_x, lc.F_aer_y, lc.F_aer_z])
    pred = sum(float(a @ b) for a, b in zip(grads, d))
    assert abs((J1 - J0) - pred) <= 1e-11 * (abs(pred) + abs(J0))
    lc.close()


def test_loads_rejects_cut_cell_on_outer_layer():
    from lsstag_b200 import _lib as L
    from lsstag_b200.loads import LoadsCalculator
    g = load_golden("loads_probe")
    lc = LoadsCalculator()
    cells = g["cells"].copy()
    cells[0] = 0                     # corner cell: its loads would read outside the grid
    with pytest.raises(L.LsgError) as e:
        lc.set(g["dims"], cells, g["type"], g["theta"], g["delta"], g["invv"], g["dmax"], g["dne"], g["dtn"],
               g["nodes"], g["center"], 2.0, 0.01)
    assert e.value.code == L.LSG_ERR_ARG
    lc.close()
