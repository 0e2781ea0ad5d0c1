"""Momentum operators assembled on the GPU from the geometry
(lsg_set_matrix_helmholtz) against the reference's own assembly
(HelmholtzDiscreteOperatorX/Y/Z): a sphere's mesh and seeded random geometry
on every cell type (flow task and non-flow task).  Entries agree to 1e-14
relative to their row (fluid and cut-cell rows bitwise); the ILU(0)-FGMRES(13)
momentum solve on the GPU-assembled operator reproduces the reference's
iterations (+-1) and solution (relative L2 <= 1e-10)."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def _geom(g, d):
    c = "xyz"[d]
    out = {k: g[k] for k in ("theta", "alpha", "delta", "inv_vof", "dib_en", "dib_ws", "dib_nb", "dib_st",
                             "inv_dib_ne", "inv_dib_tn")}
    out["stype"] = g[c + "type"]
    out["vof"] = g["vof_" + c]
    return out


def _check_planes(P, rp, col, val, dims, stype):
    import ref_runner as rr
    ref = rr.csr_to_planes(rp, col, val, dims)
    n = rp.size - 1
    scale = np.abs(ref).max(axis=0)
    err = np.abs(P - ref).max(axis=0)
    assert np.all(err <= 1e-14 * scale), float((err / np.maximum(scale, 1e-300)).max())
    inner = (stype == 11111111) | (stype > 0)
    assert np.array_equal(P[:, inner], ref[:, inner])          # fluid and cut-cell rows bitwise
    assert n == P.shape[1]


@pytest.mark.parametrize("d", [0, 1, 2])
def test_helmholtz_assembly_sphere(d):
    from lsstag_b200 import solver as S
    g = load_golden("helm_sphere16")
    nu, coef, isflow, _ = (float(v) for v in g["nu_coef_isflow_dt"])
    s = S.ILUFGMRES()
    s.set_helmholtz(d, _geom(g, d), g["dims"], nu, coef, bool(isflow), setup=False)
    k = "K" + "xyz"[d]
    _check_planes(s.planes(), g[k + "_rowptr"], g[k + "_col"], g[k + "_val"], s.dims, g["xyz"[d] + "type"])
    s.close()


@pytest.mark.parametrize("flow", [True, False])
@pytest.mark.parametrize("d", [0, 1, 2])
def test_helmholtz_assembly_random_geometry(d, flow):
    from lsstag_b200 import solver as S
    g = load_golden("helm_random14")
    nu, coef, _ = (float(v) for v in g["nu_coef_dt"])
    s = S.ILUFGMRES()
    s.set_helmholtz(d, _geom(g, d), g["dims"], nu, coef, flow, setup=False)
    k = "K" + "xyz"[d] + ("_flow" if flow else "_noflow")
    _check_planes(s.planes(), g[k + "_rowptr"], g[k + "_col"], g[k + "_val"], s.dims, g["xyz"[d] + "type"])
    s.close()


def test_momentum_solve_on_gpu_assembled_operator():
    """The reference's momentum solve (ILUFGMRES on K, its right-hand side)
    repeated with K assembled on the GPU from the geometry."""
    from lsstag_b200 import solver as S
    h = load_golden("helm_sphere16")
    g = load_golden("sphere16")
    nu, coef, isflow, _ = (float(v) for v in h["nu_coef_isflow_dt"])
    for d, c in enumerate("xyz"):
        s = S.ILUFGMRES()
        s.set_helmholtz(d, _geom(h, d), h["dims"], nu, coef, bool(isflow),
                        task=S.Task(eps=float(g[f"mom_eps_{c}"][0]), MAX_ITER=200,
                                    FGMRES_RESTART_NUM=int(g["mom_restart"][0])))
        x = np.zeros(int(np.prod(s.dims)))
        it = s.solve(g[f"mom_rhs_{c}"], x)
        assert abs(it - int(g[f"mom_it_{c}"][0])) <= 1, c
        ref = g[f"mom_x_{c}"]
        assert np.linalg.norm(x - ref) <= 1e-10 * np.linalg.norm(ref), c
        s.close()


def test_helmholtz_rejects_inconsistent_types():
    from lsstag_b200 import _lib as L
    from lsstag_b200 import solver as S
    g = load_golden("helm_sphere16")
    geom = _geom(g, 0)
    st = geom["stype"].copy()
    st[0] = 11111111             # a fluid cell in the corner keeps faces outside the grid
    geom["stype"] = st
    s = S.ILUFGMRES()
    with pytest.raises(L.LsgError) as e:
        s.set_helmholtz(0, geom, g["dims"], 0.01, 150.0, True, setup=False)
    assert e.value.code == L.LSG_ERR_ARG
    s.close()


@pytest.mark.parametrize("d", [0, 1, 2])
def test_helmholtz_flux_bitwise(d):
    """Boundary source term, then the immersed-boundary term written over it,
    on seeded random geometry, cell sizes and boundary velocities: bitwise."""
    from lsstag_b200 import solver as S
    g = load_golden("helm_random14")
    c = "xyz"[d]
    nu = float(g["nu_coef_dt"][0])
    s = S.ILUFGMRES()
    f = s.helmholtz_flux(d, g["dims"], g[c + "type"], g["delta"], g["u_w"], g["bc"], nu)
    assert np.array_equal(f, g["hflux_" + c])
    keys = ("side_type", "theta", "alpha", "inv_vof", "dib_en", "dib_ws", "dib_nb", "dib_st", "inv_dib_ne",
            "inv_dib_tn", "vib", "vibyx", "vibzy")
    fi = s.helmholtz_flux(d, g["dims"], g[c + "type"], g["delta"], g["u_w"], g["bc"], nu,
                          ib_geom={k: g[k] for k in keys})
    assert np.array_equal(fi, g["hflux_ib_" + c])
    s.close()


def test_helmholtz_flux_on_sphere_matches_momentum_step_input():
    """The source term the reference's momentum step used (the hflux input
    of lsg_momentum_rhs in the momentum-step fixture) from the geometry."""
    from lsstag_b200 import solver as S
    h = load_golden("helm_sphere16")
    g = load_golden("sphere16")
    nu = float(h["nu_coef_isflow_dt"][0])
    s = S.ILUFGMRES()
    for d, c in enumerate("xyz"):
        f = s.helmholtz_flux(d, h["dims"], h[c + "type"], h["delta"], h["u_w"], h["bc"], nu)
        assert np.array_equal(f, g["mstep_hflux_" + c]), c
    s.close()


@pytest.mark.parametrize("d", [0, 1, 2])
def test_convective_flux_bitwise(d):
    from lsstag_b200 import solver as S
    g = load_golden("helm_random14")
    s = S.ILUFGMRES()
    f = s.convective_flux(d, g["dims"], g["theta"], g["delta"], g["ux"], g["uy"], g["uz"], g["u_w"], g["bc"])
    assert np.array_equal(f, g["cflux_" + "xyz"[d]])
    s.close()


def test_convective_flux_sphere_is_the_momentum_step_input():
    from lsstag_b200 import solver as S
    h = load_golden("helm_sphere16")
    g = load_golden("sphere16")
    s = S.ILUFGMRES()
    for d, c in enumerate("xyz"):
        f = s.convective_flux(d, h["dims"], h["theta"], h["delta"], g["mstep_u_x"], g["mstep_u_y"], g["mstep_u_z"],
                              h["u_w"], h["bc"])
        assert np.array_equal(f, g["flux2_1" + c]), c
    s.close()
