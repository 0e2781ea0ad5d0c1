"""Generate the golden fixtures in this directory from the reference's own
solver (oracle/_ref/ref_harness, built by oracle/build_ref.sh from the
reference sources).  Run from the repository root:

    python tests/golden/make_golden.py

Each fixture is a compressed .npz holding the case's Laplace CSR exactly as
the reference assembles it (laplace_discrete_operator.h), the seeded
right-hand side, and the reference's outputs: its multigrid hierarchy
(P, R, A_H, factored ADLJ tridiagonals), one V-cycle, one MG-FGMRES(30) solve
and one ILU(0)-BiCGStab solve to a 1e-10 relative residual; the projection
operators (divergence Dx/Dy/Dz, gradient Gx/Gy/Gz, staggered cell types) and
one pressure projection of the time step (right-hand side, MG-FGMRES pressure
correction, corrected u, v, w, p) on seeded predicted fields; the momentum
operators (Helmholtz Kx/Ky/Kz, convective Cx/Cy/Cz) and one ILU-FGMRES solve
of each Helmholtz system; the pressure-equation source term (flux) with
nonzero boundary and immersed-boundary velocities.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "ls-stag-3d_parallel_b200"))

import lsg_oracle as lo  # noqa: E402
import ref_runner as rr  # noqa: E402
from lsstag_b200 import synth  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def cases():
    """(name, Case, rhs seed).  Small grids whose coarsening visits the
    even-even-even, even-even-odd and odd-odd-odd transfer classes."""
    out = []
    h = 1.0 / 16
    out.append(("sphere16", rr.Case(16, 16, 16, h, h, h,
                                    spheres=[(0.5 + 0.3 * h, 0.5 + 0.2 * h, 0.5 + 0.1 * h, 0.18)]), 5))
    h = 1.0 / 20
    out.append(("sphere20x12x10", rr.Case(20, 12, 10, h, h, h,
                                          spheres=[(0.5 + 0.3 * h, 0.3 + 0.2 * h, 0.25 + 0.1 * h, 0.09)]), 6))
    h = 1.0 / 24
    sph = synth.four_spheres(3, rmin=0.05, rmax=0.1, cmin=0.4, cmax=0.6)
    out.append(("spheres4_24", rr.Case(24, 24, 24, h, h, h, spheres=sph), 7))
    return out


def main():
    if not rr.available():
        sys.exit("oracle/_ref/ref_harness missing: run oracle/build_ref.sh first")
    for name, case, seed in cases():
        g = rr.run(case, threads=1)
        rp, col, val, dims = rr.csr(g, "A")
        mask = synth.connected_fluid(rp, col, val, g["pins"])
        b = synth.poisson_rhs(seed, g["celltype"], g["pins"], mask)
        r = rr.run(case, b, threads=1, fgmres=1, bicgstab=1, dump_mg=1, dump_geometry=0,
                   restart=30, rel_tol=1e-10, max_it=200)
        keep = {"dims": np.array(dims), "A_rowptr": rp, "A_col": col, "A_val": val,
                "theta": g["theta"], "delta": g["delta"], "inv_mx": g["inv_mx"], "inv_my": g["inv_my"],
                "inv_mz": g["inv_mz"], "flux": g["flux"],
                "pins": g["pins"], "celltype": g["celltype"], "b": b, "eps": r["eps"],
                "vcycle_x": r["vcycle_x"], "fgmres_x": r["fgmres_x"], "fgmres_it": r["fgmres_it"],
                "fgmres_norm_r": r["fgmres_norm_r"], "bicgstab_x": r["bicgstab_x"],
                "bicgstab_it": r["bicgstab_it"], "bicgstab_norm_r": r["bicgstab_norm_r"],
                "mg_nlev": r["mg_nlev"]}
        # one pressure projection on seeded predicted velocities and pressure
        N, M, K = dims
        gp = rr.run(case, threads=1, dump_projection=1)
        rng = np.random.default_rng(100 + seed)
        pu = 1.0 + 0.1 * rng.standard_normal((N - 1) * M * K)
        pv = 0.1 * rng.standard_normal(N * (M - 1) * K)
        pw = 0.1 * rng.standard_normal(N * M * (K - 1))
        pp = rng.standard_normal(N * M * K)
        D = tuple(rr.csr(gp, k)[:3] for k in ("Dx", "Dy", "Dz"))
        bproj = lo.projection_rhs(D, pu, pv, pw, gp["flux"], gp["pins"])
        pr = rr.run_projection(case, pu, pv, pw, pp, 1e-10 * float(np.linalg.norm(bproj)))
        for k in ("xtype", "ytype", "ztype"):
            keep[k] = gp[k]
        for m in ("Dx", "Dy", "Dz", "Gx", "Gy", "Gz"):
            for part in ("rowptr", "col", "val"):
                keep[f"{m}_{part}"] = gp[f"{m}_{part}"]
        keep.update(proj_u_in=pu, proj_v_in=pv, proj_w_in=pw, proj_p_in=pp)
        for k in ("proj_b", "proj_phi", "proj_it", "proj_u_out", "proj_v_out", "proj_w_out", "proj_p_out", "proj_coef",
                  "proj_vbase"):
            keep[k] = pr[k]
        # the momentum equations: Helmholtz and convective operators on the
        # staggered grids and one ILU-FGMRES solve of each Helmholtz system
        # (right-hand side zero on solid staggered cells, like the pressure one)
        mrhs = [rng.standard_normal((N - 1) * M * K) * (gp["xtype"] != 0),
                rng.standard_normal(N * (M - 1) * K) * (gp["ytype"] != 0),
                rng.standard_normal(N * M * (K - 1)) * (gp["ztype"] != 0)]
        mr = rr.run_momentum(case, mrhs, mom_step=1)
        for d, rhs_d in zip("xyz", mrhs):
            for m in ("K", "C"):
                for part in ("rowptr", "col", "val", "dims"):
                    keep[f"{m}{d}_{part}"] = mr[f"{m}{d}_{part}"]
            keep[f"mom_rhs_{d}"] = rhs_d
            for k in ("mom_x_", "mom_it_", "mom_eps_"):
                keep[k + d] = mr[k + d]
        keep["mom_restart"] = mr["mom_restart"]
        # one momentum step of each equation on perturbed velocities and
        # pressure: the state from set(), the inputs, the reference's
        # right-hand side and solution
        # (the operators K and C0 of that step are the Kx.. and Cx.. above;
        # kept for the two smaller cases only, to bound the fixture size)
        if name != "spheres4_24":
            keep["mstep_p"] = mr["mstep_p"]
            keep["mstep_coef2"] = mr["mstep_coef2"]
        for d in ("xyz" if name != "spheres4_24" else ""):
            for part in ("rowptr", "col", "val", "dims"):
                keep[f"C1{d}_{part}"] = mr[f"C1{d}_{part}"]
            for k in ("flux2_0", "u0", "flux2_1"):
                keep[k + d] = mr[k + d]
            for k in ("mstep_u_", "mstep_uprev_", "mstep_vof_", "mstep_hflux_", "mstep_rhs_", "mstep_sol_",
                      "mstep_it_"):
                keep[k + d] = mr[k + d]
        # the pressure-equation source term with every contribution nonzero
        # (harness flux_perturb: inflow profile, wall and immersed-boundary
        # velocities, outflow u)
        gf = rr.run(case, threads=1, flux_perturb=1)
        for k in ("side_type", "vib", "u_w", "bc_ue_vs_vn_wb_wt", "ux0", "flux"):
            keep["fluxp_" + k] = gf[k]
        for l in range(int(r["mg_nlev"][0])):
            for m in ("P", "R", "AH"):
                for part in ("rowptr", "col", "val", "dims"):
                    keep[f"mg{l}_{m}_{part}"] = r[f"mg{l}_{m}_{part}"]
            keep[f"mg{l}_odd"] = r[f"mg{l}_odd"]
            for d in "xyz":
                for part in "cde":
                    keep[f"mg{l}_{d}{part}"] = r[f"mg{l}_{d}{part}"]
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **keep)
        print(f"{path}: n={len(b)} fgmres_it={int(r['fgmres_it'][0])} "
              f"bicgstab_it={int(r['bicgstab_it'][0])} size={os.path.getsize(path)} B")


if __name__ == "__main__":
    main()
