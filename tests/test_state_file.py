"""The reference's continue-state file (SetSolutions::saveState / load):
the file the reference wrote after two time steps parses into the states
of those steps, and writing it back gives the same bytes."""
import os
import tempfile

import numpy as np

from conftest import load_golden


def test_reference_state_file_roundtrip():
    from lsstag_b200 import state as S
    f = load_golden("flow16_state")
    g = load_golden("flow16_steps")
    raw = f["state_bytes"].tobytes()
    d = tempfile.mkdtemp()
    path = os.path.join(d, "continue.dat")
    with open(path, "wb") as fh:
        fh.write(raw)
    st = S.read_state(path, g["dims"])
    assert st.it == int(f["state_it"][0]) and st.time == float(f["state_time"][0])
    for a, k in zip(st.current, ("u_2", "v_2", "w_2", "p_2")):
        assert np.array_equal(a, g[k])
    for a, k in zip(st.previous, ("u_1", "v_1", "w_1", "p_1")):
        assert np.array_equal(a, g[k])
    S.write_state(path + ".out", st)
    with open(path + ".out", "rb") as fh:
        assert fh.read() == raw
    # a truncated file is rejected, not misread
    with open(path + ".cut", "wb") as fh:
        fh.write(raw[:-8])
    try:
        S.read_state(path + ".cut", g["dims"])
    except ValueError:
        pass
    else:
        raise AssertionError("truncated state file accepted")
