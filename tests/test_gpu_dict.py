"""The row-dictionary build on the GPU (hash table, scan-numbered classes in
first-seen order) against a first-seen dedup on the host (numpy), bit for
bit, on the fine operator; on every coarse Galerkin level the classes are
checked for the dictionary's invariants (distinct rows, first-seen
numbering).  The setup wall times are reported."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def _first_seen(rows):
    """(cls, table) of a serial first-seen dedup of the rows (bitwise)."""
    rows = np.ascontiguousarray(rows)
    v = rows.view(np.dtype((np.void, rows.dtype.itemsize * rows.shape[1]))).ravel()
    _, idx, inv = np.unique(v, return_index=True, return_inverse=True)
    order = np.argsort(idx)
    rank = np.empty_like(order)
    rank[order] = np.arange(order.size)
    return rank[inv.ravel()].astype(np.int32), rows[idx[order]]


def _check_invariants(cls, table):
    n = cls.size
    assert cls.min() == 0 and cls.max() == table.shape[0] - 1
    _, first = np.unique(cls, return_index=True)
    assert np.all(np.diff(first) > 0)                     # class k first seen before class k + 1
    tv = np.ascontiguousarray(table).view(np.dtype((np.void, 8 * table.shape[1]))).ravel()
    assert np.unique(tv).size == table.shape[0]            # the rows are distinct
    assert n >= table.shape[0]


@pytest.mark.parametrize("case", ["sphere16", "128"])
def test_device_dictionary_equals_first_seen_dedup(case):
    from lsstag_b200 import cases
    from lsstag_b200 import solver as S
    from ref_runner import csr_to_planes
    if case == "sphere16":
        g = load_golden("sphere16")
        dims = tuple(int(v) for v in g["dims"])
        P = csr_to_planes(g["A_rowptr"], g["A_col"], g["A_val"], dims)
    else:
        P, dims, pins, b = cases.load(128)
    s = S.MGFGMRES()
    s.set_planes(P, dims, S.Task())
    cls, table = s.row_classes(0)
    rcls, rtable = _first_seen(np.ascontiguousarray(P.T))
    assert np.array_equal(cls, rcls)
    assert table.tobytes() == rtable.tobytes()
    levels = s.num_levels()
    for lv in range(1, levels + 1):
        c, t = s.row_classes(lv)
        assert c.size == int(np.prod(s.level_dims(lv)))
        _check_invariants(c, t)
    mms, sms = s.setup_times()
    print(f"{case}: {table.shape[0]} distinct fine rows of {cls.size}; operator + dictionary {mms:.1f} ms, "
          f"setup {sms:.1f} ms")
    assert mms > 0 and sms > 0
    s.close()


def test_all_distinct_rows():
    """An operator whose rows are all different (every coefficient perturbed,
    as on a stretched mesh): one class per row, numbered in row order, and
    the solve matches the plane-form apply."""
    from lsstag_b200 import solver as S
    g = load_golden("sphere16")
    dims = tuple(int(v) for v in g["dims"])
    from ref_runner import csr_to_planes
    P = csr_to_planes(g["A_rowptr"], g["A_col"], g["A_val"], dims)
    rng = np.random.default_rng(7)
    Q = P * (1.0 + 1e-3 * rng.random(P.shape)) * (P != 0)
    empty = np.abs(Q).sum(axis=0) == 0                     # the pinned rows: give them distinct diagonals
    Q[3, empty] = 1.0 + rng.random(int(empty.sum()))
    s = S.MGFGMRES()
    s.set_planes(Q, dims, S.Task(eps=1e-10))
    cls, table = s.row_classes(0)
    n = cls.size
    assert table.shape[0] == n and np.array_equal(cls, np.arange(n, dtype=np.int32))
    assert table.tobytes() == np.ascontiguousarray(Q.T).tobytes()
    x = rng.standard_normal(n)
    y = s.apply(x)
    # the product of the same operator in CSR form
    import scipy.sparse as sp
    from lsstag_b200.cases import planes_to_csr
    rp, col, val = planes_to_csr(Q, dims)
    A = sp.csr_matrix((val, col, rp), shape=(n, n))
    assert np.linalg.norm(y - A @ x) <= 1e-12 * np.linalg.norm(y)
    s.close()
