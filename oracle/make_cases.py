"""TEST INFRASTRUCTURE: generate the four-sphere case files
(ls-stag-3d_parallel_b200/cases/spheres4_seed3_<n>.npz) from the reference's
own geometry and Laplace-operator assembly (oracle/_ref/ref_harness, built by
oracle/build_ref.sh): the operator's seven coefficient planes exactly as the
reference's CSR holds them (signed zeros included), the pinned rows and the
solid-cell mask.  The product builds the same operator on the GPU from the
seeded spheres (lsstag_b200.cases.build_on_device); the files are the
reference side of that comparison and the reference arm's input.  Run from
the repository root:

    python oracle/make_cases.py 128 256
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "ls-stag-3d_parallel_b200"))

import ref_runner as rr  # noqa: E402
from lsstag_b200 import cases, synth  # noqa: E402


def main(sizes, seed=3):
    for n in sizes:
        h = 1.0 / n
        case = rr.Case(n, n, n, h, h, h, spheres=synth.four_spheres(seed))
        # the Laplace operator alone (operator_only: no solver set-up) and the
        # mesh build's cell types
        g = rr.run(case, threads=os.cpu_count() or 1, operator_only=1, timeout=7200)
        m = rr.run(case, threads=os.cpu_count() or 1, mesh_dump=1, timeout=7200)
        rp, col, val, dims = rr.csr(g, "A")
        P = rr.csr_to_planes(rp, col, val, dims)
        g["celltype"] = m["celltype"]
        path = cases.case_path(n, seed)
        np.savez_compressed(path, planes=P, dims=np.array(dims), pins=g["pins"],
                            solid=(g["celltype"] == 0), seed=np.array([seed]),
                            spheres=np.array(synth.four_spheres(seed)))
        print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main([int(a) for a in sys.argv[1:]] or [128, 256])
