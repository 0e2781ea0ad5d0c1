"""Generate tecplot16.npz in this directory from the reference's own code
(oracle/_ref/ref_harness, built by oracle/build_ref.sh): one time step of the
16^3 sphere flow (the flow16_steps case) and the Tecplot solution file the
reference's SolTecplotPrinter prints for the resulting state, byte for byte,
with that state (u, v, w, p) and the mesh's cell-centre nodes.  Run from the
repository root:

    python tests/golden/make_tecplot_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import ref_runner as rr  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    if not rr.available():
        sys.exit("oracle/_ref/ref_harness missing: run oracle/build_ref.sh first")
    h = 1.0 / 16
    case = rr.Case(16, 16, 16, h, h, h, spheres=[(0.5 + 0.3 * h, 0.5 + 0.2 * h, 0.5 + 0.1 * h, 0.18)])
    r = rr.run(case, threads=1, flow_steps=1, restart=30, dump_geometry=0, timeout=600, print_sol=1)
    g = np.load(os.path.join(HERE, "flow16_steps.npz"))
    for k in ("celltype", "theta", "delta", "u_w", "bc"):
        assert np.array_equal(np.asarray(r[k]).ravel(), np.asarray(g[k]).ravel()), k
    keep = {"sol": np.asarray(r["sol_bytes"], dtype=np.uint8), "nodes": r["nodes"],
            "u": r["u_1"], "v": r["v_1"], "w": r["w_1"], "p": r["p_1"]}
    path = os.path.join(HERE, "tecplot16.npz")
    np.savez_compressed(path, **keep)
    print(path, os.path.getsize(path))


if __name__ == "__main__":
    main()
