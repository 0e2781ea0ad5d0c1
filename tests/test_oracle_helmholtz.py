"""The CPU restatement of the momentum operators (HelmholtzDiscreteOperator
X/Y/Z, helmholtz_discrete_operator_*.h) against the reference's own
assembly: a sphere's mesh, and seeded random geometry on every cell type as
a flow task and as a task that is not a flow.  Bitwise."""
import numpy as np
import pytest

from conftest import load_golden

import lsg_oracle as O


def _assemble(g, d, is_flow, nu, coef):
    N, M, K = (int(v) for v in g["dims"])
    c = "xyz"[d]
    return O.helmholtz_from_geometry(d, N, M, K, g[c + "type"], g["theta"], g["alpha"], g["delta"], g["inv_vof"],
                                     g["vof_" + c], g["dib_en"], g["dib_ws"], g["dib_nb"], g["dib_st"],
                                     g["inv_dib_ne"], g["inv_dib_tn"], nu, coef, is_flow)


@pytest.mark.parametrize("d", [0, 1, 2])
def test_helmholtz_sphere_bitwise(d):
    g = load_golden("helm_sphere16")
    nu, coef, isflow, _ = g["nu_coef_isflow_dt"]
    rp, col, val = _assemble(g, d, bool(isflow), nu, coef)
    k = "K" + "xyz"[d]
    assert np.array_equal(rp, g[k + "_rowptr"]) and np.array_equal(col, g[k + "_col"])
    assert np.array_equal(val, g[k + "_val"])


@pytest.mark.parametrize("flow", [True, False])
@pytest.mark.parametrize("d", [0, 1, 2])
def test_helmholtz_random_geometry_bitwise(d, flow):
    g = load_golden("helm_random14")
    nu, coef, _ = g["nu_coef_dt"]
    rp, col, val = _assemble(g, d, flow, nu, coef)
    k = "K" + "xyz"[d] + ("_flow" if flow else "_noflow")
    assert np.array_equal(rp, g[k + "_rowptr"]) and np.array_equal(col, g[k + "_col"])
    assert np.array_equal(val, g[k + "_val"])
    # every box-boundary family, fluid, solid and cut cells are present
    types = set(int(t) for t in g["xyz"[d] + "type"])
    assert set(range(-27, -1)) <= types and {0, 11111111} <= types and any(t > 0 and t != 11111111 for t in types)


@pytest.mark.parametrize("d", [0, 1, 2])
def test_helmholtz_flux_bitwise(d):
    g = load_golden("helm_random14")
    N, M, K = (int(v) for v in g["dims"])
    nu = float(g["nu_coef_dt"][0])
    c = "xyz"[d]
    f = O.helmholtz_flux(d, N, M, K, g[c + "type"], g["delta"], g["u_w"], g["bc"], nu)
    assert np.array_equal(f, g["hflux_" + c])
    fi = O.helmholtz_ib_flux(d, N, M, K, g[c + "type"], g["side_type"], g["theta"], g["alpha"], g["delta"],
                             g["inv_vof"], g["dib_en"], g["dib_ws"], g["dib_nb"], g["dib_st"], g["inv_dib_ne"],
                             g["inv_dib_tn"], g["vib"], g["vibyx"], g["vibzy"], nu, f)
    assert np.array_equal(fi, g["hflux_ib_" + c])
    assert np.count_nonzero(fi != f) > 0            # the immersed-boundary rows changed


def test_helmholtz_flux_sphere_is_the_momentum_step_input():
    """On the sphere case the restated source term equals the hflux the
    reference's momentum step used (momentum-step fixture)."""
    h = load_golden("helm_sphere16")
    g = load_golden("sphere16")
    N, M, K = (int(v) for v in h["dims"])
    nu = float(h["nu_coef_isflow_dt"][0])
    for d, c in enumerate("xyz"):
        f = O.helmholtz_flux(d, N, M, K, h[c + "type"], h["delta"], h["u_w"], h["bc"], nu)
        assert np.array_equal(f, g["mstep_hflux_" + c]), c


@pytest.mark.parametrize("d", [0, 1, 2])
def test_convective_flux_bitwise(d):
    """Source term of the convective operators (0 for x and y, as the
    reference leaves it) on seeded geometry, velocities and boundary values."""
    g = load_golden("helm_random14")
    N, M, K = (int(v) for v in g["dims"])
    f = O.convective_flux(d, N, M, K, g["theta"], g["delta"], g["ux"], g["uy"], g["uz"], g["u_w"], g["bc"])
    assert np.array_equal(f, g["cflux_" + "xyz"[d]])
    if d == 2:
        assert np.count_nonzero(f) > 0


def test_convective_flux_sphere_is_the_momentum_step_input():
    h = load_golden("helm_sphere16")
    g = load_golden("sphere16")
    for d, c in enumerate("xyz"):
        f = O.convective_flux(d, 16, 16, 16, h["theta"], h["delta"], g["mstep_u_x"], g["mstep_u_y"], g["mstep_u_z"],
                              h["u_w"], h["bc"])
        assert np.array_equal(f, g["flux2_1" + c]), c
