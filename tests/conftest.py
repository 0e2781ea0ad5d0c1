import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "oracle"), os.path.join(ROOT, "ls-stag-3d_parallel_b200"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


GOLDEN = os.path.join(ROOT, "tests", "golden")
GOLDEN_CASES = ["sphere16", "sphere20x12x10", "spheres4_24"]


def load_golden(name):
    import numpy as np
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def golden_csr(g, prefix="A"):
    import scipy.sparse as sp
    rp, col, val = g[prefix + "_rowptr"], g[prefix + "_col"], g[prefix + "_val"]
    n = rp.size - 1
    ncol = int(col.max()) + 1 if col.size else n
    return sp.csr_matrix((val, col, rp), shape=(n, max(n, ncol)))
