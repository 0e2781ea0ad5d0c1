"""Generate the four-sphere case files of this directory from the reference's
own geometry and Laplace-operator assembly (oracle/_ref/ref_harness, built by
oracle/build_ref.sh).  Run from the repository root:

    python ls-stag-3d_parallel_b200/cases/make_cases.py 128 256
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "ls-stag-3d_parallel_b200"))

import ref_runner as rr  # noqa: E402
from lsstag_b200 import cases, synth  # noqa: E402


def main(sizes, seed=3):
    for n in sizes:
        h = 1.0 / n
        case = rr.Case(n, n, n, h, h, h, spheres=synth.four_spheres(seed))
        g = rr.run(case, threads=os.cpu_count() or 1, dump_geometry=1)
        rp, col, val, dims = rr.csr(g, "A")
        P = rr.csr_to_planes(rp, col, val, dims)
        path = cases.case_path(n, seed)
        np.savez_compressed(path, planes=P, dims=np.array(dims), pins=g["pins"],
                            solid=(g["celltype"] == 0), seed=np.array([seed]),
                            spheres=np.array(synth.four_spheres(seed)))
        print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main([int(a) for a in sys.argv[1:]] or [128, 256])
