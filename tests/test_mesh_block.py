"""Host logic of the device mesh build (CPU): the level-set block rule and
the body records reproduce what the reference's mesh build used for every
golden mesh case (tests/golden/mesh_*.npz, dumped by the reference)."""
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN

CASES = sorted(glob.glob(os.path.join(GOLDEN, "mesh_*.npz")))


def _bodies(g):
    from lsstag_b200 import mesh as MS
    sph = [tuple(s) for s in g["spheres"].reshape(-1, 4)]
    ell = [(e[0:3], e[3:6], e[6:15].reshape(3, 3)) for e in g["ellipsoids"].reshape(-1, 15)]
    return sph, ell, MS.bodies_array(sph, ell)


@pytest.mark.parametrize("path", CASES, ids=[os.path.basename(p)[5:-4] for p in CASES])
def test_flow_block_matches_reference(path):
    from lsstag_b200 import mesh as MS
    g = dict(np.load(path))
    sph, ell, recs = _bodies(g)
    assert recs.shape == (len(sph) + len(ell), MS.BODY_WORDS)
    assert tuple(MS.flow_block(g["dims"], g["h"], sph, ell)) == tuple(int(v) for v in g["ls_block"])


def test_field_sizes():
    from lsstag_b200 import mesh as MS
    dims = (5, 4, 3)
    assert MS.field_size("alpha", dims) == 180
    assert MS.field_size("inv_mx", dims) == 4 * 4 * 3
    assert MS.field_size("ytype", dims) == 5 * 3 * 3
    assert MS.field_size("vof_z", dims) == 5 * 4 * 2
