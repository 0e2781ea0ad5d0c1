"""Generate tests/golden/mixed12x10x8.npz from the reference's own solver
(oracle/_ref/ref_harness).  Run from the repository root:

    python tests/golden/make_mixed_parity_golden.py

A 12 x 10 x 8 sphere case whose second coarsening (6 x 5 x 4 -> 3 x 3 x 2)
is the even-odd-even transfer class: the fixture holds the reference's
Laplace CSR, a seeded right-hand side, its multigrid hierarchy (P, R, A_H of
both coarsenings), one V-cycle and one MG-FGMRES(30) solve to 1e-10."""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "ls-stag-3d_parallel_b200"))

import ref_runner as rr  # noqa: E402
from lsstag_b200 import synth  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    if not rr.available():
        sys.exit("oracle/_ref/ref_harness missing: run oracle/build_ref.sh first")
    h = 1.0 / 12
    case = rr.Case(12, 10, 8, h, h, h, spheres=[(0.5 + 0.3 * h, 0.42 + 0.2 * h, 0.33 + 0.1 * h, 0.15)])
    g = rr.run(case, threads=1)
    rp, col, val, dims = rr.csr(g, "A")
    mask = synth.connected_fluid(rp, col, val, g["pins"])
    b = synth.poisson_rhs(8, g["celltype"], g["pins"], mask)
    r = rr.run(case, b, threads=1, fgmres=1, bicgstab=0, dump_mg=1, dump_geometry=0, restart=30, rel_tol=1e-10,
               max_it=200)
    keep = {"dims": np.array(dims), "A_rowptr": rp, "A_col": col, "A_val": val, "pins": g["pins"], "b": b,
            "eps": r["eps"], "vcycle_x": r["vcycle_x"], "fgmres_x": r["fgmres_x"], "fgmres_it": r["fgmres_it"],
            "fgmres_norm_r": r["fgmres_norm_r"], "mg_nlev": r["mg_nlev"]}
    for l in range(int(r["mg_nlev"][0])):
        for k in ("P", "R", "AH"):
            for part in ("rowptr", "col", "val", "dims"):
                keep[f"mg{l}_{k}_{part}"] = r[f"mg{l}_{k}_{part}"]
    out = os.path.join(HERE, "mixed12x10x8.npz")
    np.savez_compressed(out, **keep)
    print(out, os.path.getsize(out))


if __name__ == "__main__":
    main()
