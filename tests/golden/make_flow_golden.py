"""Generate the time-stepping fixture in this directory from the reference's
own time step (oracle/_ref/ref_harness, built by oracle/build_ref.sh).  Run
from the repository root:

    python tests/golden/make_flow_golden.py

flow16_steps.npz: the flow past the 16^3 sphere of the other fixtures
(uniform inflow U = 1, the flow task's walls and outflow, Re 100, dt 0.01),
three time steps as TimeSteppingMethodInterface::step runs them (momentum
equations, pressure equation, projection) with absolute solver tolerance
1e-11 and no start-up pressure scaling; every mesh array the GPU path reads,
the initial state, and per step the predicted velocities, the pressure
correction, the iteration counts and the new state.

flow16_state.npz: the reference's own continue-state file
(SetSolutions::saveState) after the first two of those steps, byte for byte.
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
    r = rr.run(case, threads=1, flow_steps=3, task_eps=1e-11, restart=30, dump_geometry=0)
    np.savez_compressed(os.path.join(HERE, "flow16_steps.npz"), **r)
    print("flow16_steps.npz", os.path.getsize(os.path.join(HERE, "flow16_steps.npz")))
    # the reference's continue-state file after two of those steps
    s = rr.run(case, threads=1, flow_steps=2, task_eps=1e-11, restart=30, dump_geometry=0, save_state=1)
    np.savez_compressed(os.path.join(HERE, "flow16_state.npz"), state_bytes=s["state_bytes"],
                        state_it=s["state_it"], state_time=s["state_time"])
    print("flow16_state.npz", os.path.getsize(os.path.join(HERE, "flow16_state.npz")))


if __name__ == "__main__":
    main()
