"""Generate tests/golden/bicgstab_band.npz: the reference's own ILU(0)-BiCGStab
(ilu_bicgstab.h, bicgstab_interface.h:76-111) on the golden Poisson systems,
solved to a 1e-10 relative residual with 1, 2, 4 and 8 OpenMP threads.
BiCGStab amplifies the summation order of its dot products, so the
reference's iteration count and solution move with the thread count; the
spread it shows against its own 1-thread run is the bar the GPU solve is
held to.  Run from the repository root (after oracle/build_ref.sh):

    python tests/golden/make_bicgstab_band.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "ls-stag-3d_parallel_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))

import ref_runner as rr  # noqa: E402
from make_golden import cases  # noqa: E402

THREADS = (1, 2, 4, 8)


def main():
    out = {"threads": np.array(THREADS)}
    for name, case, _seed in cases():
        g = np.load(os.path.join(ROOT, "tests", "golden", f"{name}.npz"))
        its, xs = [], []
        for th in THREADS:
            r = rr.run(case, g["b"], threads=th, fgmres=0, bicgstab=1, dump_geometry=0, restart=30, rel_tol=1e-10,
                       max_it=200)
            its.append(int(r["bicgstab_it"][0]))
            xs.append(r["bicgstab_x"])
        x1 = xs[0]
        assert np.array_equal(x1, g["bicgstab_x"]), name     # the fixture's 1-thread solve
        spread = [float(np.linalg.norm(x - x1) / np.linalg.norm(x1)) for x in xs]
        out[f"{name}_its"] = np.array(its)
        out[f"{name}_spread"] = np.array(spread)
        print(name, "iterations", its, "rel L2 to the 1-thread solve", spread)
    np.savez(os.path.join(ROOT, "tests", "golden", "bicgstab_band.npz"), **out)


if __name__ == "__main__":
    main()
