"""The CPU restatement of the cut-cell loads (LoadsCalculator,
loads_calculator.h) against the reference's own outputs: every cut-cell type
on seeded arrays (loads_probe.npz) and calculate() on a sphere's cut cells
(loads_sphere16.npz).  Per-cell forces and moments are bitwise equal; sums
differ by summation order only."""
import numpy as np
import pytest

from conftest import load_golden

import lsg_oracle as O


def _probe_forces(g, nucell=None):
    N, M, K = (int(v) for v in g["dims"])
    return O.loads_forces(N, M, K, g["cells"], g["type"], g["theta"], g["delta"], g["invv"], g["dmax"],
                          g["dne"], g["dtn"], g["vib"], g["vibyx"], g["vibzy"], g["ux"], g["uy"], g["uz"],
                          g["p"], float(g["nu"]), nu_cell=nucell)


@pytest.mark.parametrize("per_cell_nu", [False, True])
def test_loads_every_cell_type_bitwise(per_cell_nu):
    g = load_golden("loads_probe")
    sfx = "_nucell" if per_cell_nu else ""
    f = _probe_forces(g, g["nucell"] if per_cell_nu else None)
    for a, k in zip(f, ("fx", "fy", "fz")):
        assert np.array_equal(a, g[k + sfx]), k
    m = O.loads_moments(g["cells"], g["nodes"], g["center"], *f)
    for a, k in zip(m, ("mz", "mx", "my")):
        assert np.array_equal(a, g[k + sfx]), k
    # every type with shear terms is present, and the shear terms matter
    types = set(int(t) for t in g["type"][g["cells"]])
    assert set(O.LOADS_TERMS) <= types


def test_loads_filter_matches_reference():
    g = load_golden("loads_probe")
    flt = O.LoadsFilter(float(g["filter_dt"]))
    out = np.array([flt.step(v) for v in g["filter_in"]])
    assert np.array_equal(out, g["filter_out"])


def test_loads_calculate_on_sphere():
    r = load_golden("loads_sphere16")
    N, M, K = (int(v) for v in r["dims"])
    nu, fcoef, dt = (float(v) for v in r["nu_fcoef_dt"])
    f = O.loads_forces(N, M, K, r["cells"], r["celltype"], r["theta"], r["delta"], r["inv_vof"], r["dmax"],
                       r["dne"], r["dtn"], r["vib"], r["vibyx"], r["vibzy"], r["ux"], r["uy"], r["uz"], r["p"], nu)
    for a, k in zip(f, ("fx", "fy", "fz")):
        assert np.array_equal(a, r[k]), k
    m = O.loads_moments(r["cells"], r["nodes"], r["center"], *f)
    sums = r["sums"]
    for c in range(3):
        assert abs(f[c].sum() - sums[c]) <= 1e-13 * np.abs(f[c]).sum()
        assert abs(f[c].sum() * fcoef - sums[3 + c]) <= 1e-13 * np.abs(f[c]).sum() * fcoef
        flt = O.LoadsFilter(dt)
        assert abs(flt.step(m[c].sum()) - sums[6 + c]) <= 1e-13 * np.abs(m[c]).sum()


def test_loads_adjoint_oracle_is_the_gradient():
    """The forces are affine in (ux, uy, uz, p): J(x + d) - J(x) = <g, d>."""
    g = load_golden("loads_probe")
    N, M, K = (int(v) for v in g["dims"])
    w = np.array([1.0, -0.5, 0.25])
    grads = O.loads_adjoint(N, M, K, g["cells"], g["type"], g["theta"], g["delta"], g["invv"], g["dmax"],
                            g["dne"], g["dtn"], w, float(g["nu"]))
    rng = np.random.default_rng(2)
    f0 = _probe_forces(g)
    J0 = sum(wc * fc.sum() for wc, fc in zip(w, f0))
    d = [rng.normal(size=a.size) for a in grads]
    gg = dict(g)
    for k, dk in zip(("ux", "uy", "uz", "p"), d):
        gg[k] = g[k] + dk
    f1 = _probe_forces(gg)
    J1 = sum(wc * fc.sum() for wc, fc in zip(w, f1))
    pred = sum(float(a @ b) for a, b in zip(grads, d))
    assert abs((J1 - J0) - pred) <= 1e-12 * (abs(pred) + abs(J0))
