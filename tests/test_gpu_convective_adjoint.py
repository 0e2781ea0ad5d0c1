"""Transposed Jacobian of the convective term (lsg_convective_adjoint): the
term is bilinear in (U, v), so for any directions dU, dv
    <lam, C(dU) v + C(U) dv> = <U_bar, dU> + <v_bar, dv>
holds exactly up to rounding; checked with the forward apply on the GPU on a
sphere's mesh for all three momentum components (relative 1e-12)."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["sphere16", "spheres4_24"])
def test_convective_adjoint_dot_product(name):
    from lsstag_b200 import solver as S
    g = load_golden(name)
    dims = tuple(int(v) for v in g["dims"])
    s = S.MGFGMRES()
    s.set_geometry({k: g[k] for k in ("celltype", "theta", "delta", "inv_mx", "inv_my", "inv_mz")}, dims, g["pins"],
                   setup=False)
    s.set_staggered_types(g["xtype"], g["ytype"], g["ztype"])
    N, M, K = dims
    sizes = [(N - 1) * M * K, N * (M - 1) * K, N * M * (K - 1)]
    types = [g["xtype"], g["ytype"], g["ztype"]]
    rng = np.random.default_rng(8)
    # velocities zero inside the bodies, as the flow keeps them
    U = [np.where(t != 0, rng.standard_normal(n), 0.0) for t, n in zip(types, sizes)]
    dU = [np.where(t != 0, rng.standard_normal(n), 0.0) for t, n in zip(types, sizes)]
    for d in range(3):
        for zq in (True, False):
            v = np.where(types[d] != 0, rng.standard_normal(sizes[d]), 0.0)
            dv = np.where(types[d] != 0, rng.standard_normal(sizes[d]), 0.0)
            lam = rng.standard_normal(sizes[d])
            ub = s.convective_adjoint(d, U, v, lam, zconv_reference=zq)
            lhs = lam @ (s.convective_apply(d, dU, v, zconv_reference=zq) +
                         s.convective_apply(d, U, dv, zconv_reference=zq))
            rhs = sum(float(a @ b) for a, b in zip(ub[:3], dU)) + float(ub[3] @ dv)
            scale = sum(float(np.abs(a) @ np.abs(b)) for a, b in zip(ub[:3], dU)) + float(np.abs(ub[3]) @ np.abs(dv))
            assert abs(lhs - rhs) <= 1e-12 * scale, (d, zq, lhs, rhs)
    s.close()
