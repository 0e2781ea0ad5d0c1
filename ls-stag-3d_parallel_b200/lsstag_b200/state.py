"""The reference's continue-state file (SetSolutions::saveState / load,
Base/set_solutions.h:247-266 and :318-337): the iteration counter and time,
the centre and centre velocity of every immersed body, the loads of every
body (BaseTaskDescription::saveState, base_task_description.h:151-170), and
the current and previous solution (Solution::saveState, solution.h:82-87:
u, v, w, p as raw FP64 arrays).  Reading a file the reference wrote lets a
run continue on the GPU; a file written here continues in the reference.
Little-endian, no padding:

    int32 it; float64 time;
    per body: float64 cur_C[3], curV_C[3]
    per body: float64 F_aer_x, F_aer_y, F_aer_z, moment_aer
    current:  float64 u[(N-1)MK], v[N(M-1)K], w[NM(K-1)], p[NMK]
    previous: the same
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class FlowState:
    it: int
    time: float
    centers: np.ndarray = field(default_factory=lambda: np.zeros((0, 3)))          # cur_C per body
    center_velocities: np.ndarray = field(default_factory=lambda: np.zeros((0, 3)))  # curV_C per body
    loads: np.ndarray = field(default_factory=lambda: np.zeros((0, 4)))            # F_aer_x, _y, _z, moment_aer
    current: tuple = ()       # (u, v, w, p)
    previous: tuple = ()      # (u, v, w, p)


def _sizes(dims):
    N, M, K = (int(v) for v in dims)
    return ((N - 1) * M * K, N * (M - 1) * K, N * M * (K - 1), N * M * K)


def read_state(path: str, dims, n_bodies: int = 1) -> FlowState:
    """Parse a continue-state file for an N x M x K base grid."""
    raw = open(path, "rb").read()
    sizes = _sizes(dims)
    expect = 4 + 8 + n_bodies * 6 * 8 + n_bodies * 4 * 8 + 2 * 8 * sum(sizes)
    if len(raw) != expect:
        raise ValueError(f"state file holds {len(raw)} bytes, {expect} expected for grid {tuple(dims)} "
                         f"with {n_bodies} bodies")
    it = int(np.frombuffer(raw, "<i4", 1, 0)[0])
    off = 4
    t = float(np.frombuffer(raw, "<f8", 1, off)[0])
    off += 8
    cv = np.frombuffer(raw, "<f8", 6 * n_bodies, off).reshape(n_bodies, 6)
    off += 48 * n_bodies
    loads = np.frombuffer(raw, "<f8", 4 * n_bodies, off).reshape(n_bodies, 4).copy()
    off += 32 * n_bodies
    sols = []
    for _ in range(2):
        fields = []
        for n in sizes:
            fields.append(np.frombuffer(raw, "<f8", n, off).copy())
            off += 8 * n
        sols.append(tuple(fields))
    return FlowState(it, t, cv[:, :3].copy(), cv[:, 3:].copy(), loads, sols[0], sols[1])


def write_state(path: str, st: FlowState) -> None:
    """Write a continue-state file the reference's SetSolutions::load reads."""
    nb = len(st.centers)
    parts = [np.array([st.it], "<i4").tobytes(), np.array([st.time], "<f8").tobytes()]
    for b in range(nb):
        parts.append(np.concatenate([np.asarray(st.centers[b], "<f8"), np.asarray(st.center_velocities[b], "<f8")])
                     .tobytes())
    for b in range(nb):
        parts.append(np.asarray(st.loads[b], "<f8").reshape(4).tobytes())
    for sol in (st.current, st.previous):
        for a in sol:
            parts.append(np.ascontiguousarray(a, "<f8").tobytes())
    with open(path, "wb") as f:
        f.write(b"".join(parts))
