"""Pressure projection on the GPU (lsg_projection_rhs / lsg_projection_correct)
against the reference's own outputs: right-hand side and corrected fields
bit for bit, pressure correction within the solver's parity bounds."""
import numpy as np
import pytest

from conftest import GOLDEN_CASES, load_golden

pytestmark = pytest.mark.gpu


def _solver(g):
    from lsstag_b200 import solver as S
    dims = tuple(int(v) for v in g["dims"])
    s = S.MGFGMRES()
    geom = {k: g[k] for k in ("celltype", "theta", "delta", "inv_mx", "inv_my", "inv_mz")}
    s.set_geometry(geom, dims, g["pins"], task=S.Task(eps=1e-10 * float(np.linalg.norm(g["proj_b"])), MAX_ITER=200,
                                                      FGMRES_RESTART_NUM=30))
    s.set_staggered_types(g["xtype"], g["ytype"], g["ztype"])
    return s


def _bits(a):
    return np.ascontiguousarray(a).view(np.int64)


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_projection_rhs_bitwise(name):
    g = load_golden(name)
    s = _solver(g)
    b = s.projection_rhs(g["proj_u_in"], g["proj_v_in"], g["proj_w_in"], g["flux"])
    assert np.array_equal(_bits(b), _bits(g["proj_b"]))
    s.close()


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_projection_correct_bitwise(name):
    g = load_golden(name)
    s = _solver(g)
    p = g["proj_p_in"].copy()
    u, v, w, p = s.projection_correct(g["proj_phi"], g["proj_u_in"], g["proj_v_in"], g["proj_w_in"], p,
                                      float(g["proj_coef"][0]), float(g["proj_vbase"][0]))
    for mine, key in ((u, "proj_u_out"), (v, "proj_v_out"), (w, "proj_w_out"), (p, "proj_p_out")):
        assert np.array_equal(_bits(mine), _bits(g[key])), key
    s.close()


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_projection_step_matches_reference(name):
    """Full projection on the GPU: right-hand side, MG-FGMRES pressure
    correction, update.  phi: reference iterations +-1 and relative L2
    <= 1e-10; velocities then agree to the same relative bound (they are linear
    in phi; the clamps act on the sign of u, identical here)."""
    g = load_golden(name)
    s = _solver(g)
    b = s.projection_rhs(g["proj_u_in"], g["proj_v_in"], g["proj_w_in"], g["flux"])
    phi = np.zeros_like(b)
    it = s.solve(b, phi)
    assert abs(it - int(g["proj_it"][0])) <= 1
    assert np.linalg.norm(phi - g["proj_phi"]) <= 1e-10 * np.linalg.norm(g["proj_phi"])
    p = g["proj_p_in"].copy()
    u, v, w, p = s.projection_correct(phi, g["proj_u_in"], g["proj_v_in"], g["proj_w_in"], p,
                                      float(g["proj_coef"][0]), float(g["proj_vbase"][0]))
    for mine, key in ((u, "proj_u_out"), (v, "proj_v_out"), (w, "proj_w_out"), (p, "proj_p_out")):
        ref = g[key]
        assert np.linalg.norm(mine - ref) <= 1e-10 * np.linalg.norm(ref), key
    s.close()


def test_geometry_rejects_inconsistent_types():
    """A fluid cell on the domain border would read faces outside the grid:
    refused on the host before any kernel runs."""
    from lsstag_b200 import _lib as L
    from lsstag_b200 import solver as S
    g = load_golden("sphere16")
    dims = tuple(int(v) for v in g["dims"])
    geom = {k: g[k].copy() for k in ("celltype", "theta", "delta", "inv_mx", "inv_my", "inv_mz")}
    geom["celltype"][0] = 11111111
    s = S.MGFGMRES()
    with pytest.raises(L.LsgError):
        s.set_geometry(geom, dims, g["pins"], setup=False)
    s.close()


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_laplace_flux_bitwise(name):
    """GPU pressure-equation source term against the reference's flux, bit for
    bit, with every contribution nonzero."""
    g = load_golden(name)
    s = _solver(g)
    f = s.laplace_flux(g["fluxp_side_type"], g["fluxp_vib"], g["fluxp_u_w"], g["fluxp_bc_ue_vs_vn_wb_wt"],
                       g["fluxp_ux0"])
    assert np.array_equal(_bits(f), _bits(g["fluxp_flux"]))
    s.close()
