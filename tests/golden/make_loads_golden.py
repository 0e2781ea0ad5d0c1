"""Generate the cut-cell loads fixtures in this directory from the
reference's own code (oracle/_ref/ref_harness, built by oracle/build_ref.sh).
Run from the repository root:

    python tests/golden/make_loads_golden.py

loads_probe.npz: every cut-cell type of the reference's CellTypes enum
(LS_STAG_Mesh/cut_cells.h, read from the reference checkout) placed on the
interior of an 8 x 8 x 8 grid with seeded geometry, velocities, pressure and
immersed-boundary velocities; the reference's per-cell forces and moments
(LoadsCalculator::calc / calcMoment*) with a scalar viscosity and with a
per-cell one, and its moment filter on a signal with a spike.

loads_sphere16.npz: LoadsCalculator::calculate on the cut cells of the
sphere16 case's mesh (the reference's own geometry arrays), with seeded
velocities, pressure and immersed-boundary velocities.
"""
from __future__ import annotations

import os
import re
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import ref_runner as rr  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
REF_ROOT = os.environ.get("REF_ROOT", "/root/reference")


def cut_cell_codes():
    """Values of the cut-cell types (positive codes other than FluidCell)."""
    src = open(os.path.join(REF_ROOT, "src", "Base", "LS_STAG_Mesh", "cut_cells.h")).read()
    vals = sorted({int(v) for v in re.findall(r"=\s*(-?\d+)", src)})
    return [v for v in vals if 0 < v < 11111111]


def probe_inputs(seed=11):
    rng = np.random.default_rng(seed)
    N = M = K = 8
    n = N * M * K
    codes = cut_cell_codes()
    interior = [x + N * (y + M * z) for z in range(1, K - 1) for y in range(1, M - 1) for x in range(1, N - 1)]
    assert len(codes) + 2 <= len(interior)
    cells = np.array(interior[: len(codes) + 2], dtype=np.int32)
    ctype = np.full(n, 11111111, dtype=np.int32)                 # FluidCell elsewhere
    ctype[cells[: len(codes)]] = codes
    ctype[cells[len(codes)]] = 11111111                            # fluid and a wall type: base terms only
    ctype[cells[len(codes) + 1]] = -4
    u3 = lambda lo, hi: rng.uniform(lo, hi, 3 * n)                # noqa: E731
    inp = dict(
        type=ctype, cells=cells,
        theta=u3(0.0, 1.0), delta=u3(0.5, 1.5), vib=u3(-0.1, 0.1), vibyx=u3(-0.2, 0.2), vibzy=u3(-0.2, 0.2),
        dne=u3(0.5, 4.0), dtn=u3(0.5, 4.0), dmax=u3(0.1, 1.0), nodes=u3(0.0, 1.0),
        center=rng.uniform(0.3, 0.7, 3), invv=rng.uniform(0.5, 3.0, n), p=rng.normal(0, 0.5, n),
        ux=rng.normal(1.0, 0.3, (N - 1) * M * K), uy=rng.normal(0, 0.3, N * (M - 1) * K),
        uz=rng.normal(0, 0.3, N * M * (K - 1)))
    nucell = rng.uniform(0.005, 0.02, n)
    return (N, M, K), inp, nucell


def main():
    if not rr.available():
        sys.exit("oracle/_ref/ref_harness missing: run oracle/build_ref.sh first")
    dims, inp, nucell = probe_inputs()
    sig = np.concatenate([np.linspace(0.1, 1.0, 20), [30.0], np.linspace(1.0, 0.5, 19)])
    r0 = rr.run_loads_probe(dims, inp, 0.01, filter_in=sig, dt=0.01)
    r1 = rr.run_loads_probe(dims, dict(inp, nucell=nucell), 0.01)
    keep = {"dims": np.array(dims, dtype=np.int32), "nu": np.array(0.01), "nucell": nucell,
            "filter_in": sig, "filter_dt": np.array(0.01), "filter_out": r0["filter_out"]}
    keep.update(inp)
    for k in ("fx", "fy", "fz", "mz", "mx", "my"):
        keep[k] = r0[k]
        keep[k + "_nucell"] = r1[k]
    np.savez_compressed(os.path.join(HERE, "loads_probe.npz"), **keep)

    h = 1.0 / 16
    case = rr.Case(16, 16, 16, h, h, h, spheres=[(0.5 + 0.3 * h, 0.5 + 0.2 * h, 0.5 + 0.1 * h, 0.18)])
    r = rr.run_loads(case)
    np.savez_compressed(os.path.join(HERE, "loads_sphere16.npz"), **r)
    for f in ("loads_probe.npz", "loads_sphere16.npz"):
        print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
