"""Generate the momentum-operator fixtures in this directory from the
reference's own operator code (oracle/_ref/ref_harness, built by
oracle/build_ref.sh).  Run from the repository root:

    python tests/golden/make_helmholtz_golden.py

helm_sphere16.npz: HelmholtzDiscreteOperatorX/Y/Z built (init -> build) on
the 16^3 sphere case of the other fixtures, with every geometry array they
read.

helm_random14.npz: the same operators on a 14^3 grid with a sphere whose face fractions,
edge fractions (15 % of them exactly 0, so that the immersed-boundary
branches run on every cell type), cell volumes and immersed-boundary
distances are seeded random numbers; the cell types are the mesh's own.
Cell sizes, boundary velocities, the inflow profile and the
immersed-boundary velocities are seeded too.  Built once as a flow task
(K*_flow) and once as a task that is not a flow (K*_noflow: no outflow
terms, T/B walls); with the boundary source term of the operators (hflux_*)
and the immersed-boundary source term written over it (hflux_ib_*,
ibFluxHelmX/Y/Z, which the reference runs for moving bodies); and, on
seeded velocities (ux, uy, uz), the convective operators' source term
(cflux_*, ConvectiveDiscreteOperatorX/Y/Z::recalc).
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import ref_runner as rr  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
GEOM = ["dims", "xtype", "ytype", "ztype", "theta", "alpha", "delta", "inv_vof", "vof_x", "vof_y", "vof_z",
        "dib_en", "dib_ws", "dib_nb", "dib_st", "inv_dib_ne", "inv_dib_tn", "nu_coef_isflow_dt"]


def ops(r, tag=""):
    out = {}
    for d in "xyz":
        for part in ("rowptr", "col", "val"):
            out[f"K{d}{tag}_{part}"] = r[f"K{d}_{part}"]
    return out


def main():
    if not rr.available():
        sys.exit("oracle/_ref/ref_harness missing: run oracle/build_ref.sh first")
    h = 1.0 / 16
    case = rr.Case(16, 16, 16, h, h, h, spheres=[(0.5 + 0.3 * h, 0.5 + 0.2 * h, 0.5 + 0.1 * h, 0.18)])
    r = rr.run(case, threads=1, helm=1, dump_geometry=0)
    keep = {k: r[k] for k in GEOM + ["bc", "u_w"]}
    keep.update(ops(r))
    np.savez_compressed(os.path.join(HERE, "helm_sphere16.npz"), **keep)

    h = 1.0 / 14
    case = rr.Case(14, 14, 14, h, h, h, spheres=[(0.5 + 0.3 * h, 0.5 + 0.2 * h, 0.5 + 0.1 * h, 0.12)])
    r1 = rr.run(case, threads=1, helm=1, helm_random=1, helm_ibflux=1, helm_conv=1, seed=5, dump_geometry=0)
    r2 = rr.run(case, threads=1, helm=1, helm_random=1, helm_ibflux=1, helm_noflow=1, seed=5, dump_geometry=0)
    extra = ["side_type", "vib", "vibyx", "vibzy", "u_w", "bc"]
    for k in GEOM[:-1] + extra:
        assert np.array_equal(r1[k], r2[k]), k
    keep = {k: r1[k] for k in GEOM[:-1] + extra}
    keep["nu_coef_dt"] = r1["nu_coef_isflow_dt"][[0, 1, 3]]
    keep.update(ops(r1, "_flow"))
    keep.update(ops(r2, "_noflow"))
    for d in "xyz":
        # the source term is the same for both task kinds at build time
        assert np.array_equal(r1["hflux_" + d], r2["hflux_" + d])
        keep["hflux_" + d] = r1["hflux_" + d]
        keep["hflux_ib_" + d] = r1["hflux_ib_" + d]
        keep["cflux_" + d] = r1["cflux_" + d]
        keep["u" + d] = r1["u" + d]
    np.savez_compressed(os.path.join(HERE, "helm_random14.npz"), **keep)
    for f in ("helm_sphere16.npz", "helm_random14.npz"):
        print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
