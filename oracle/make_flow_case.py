"""TEST INFRASTRUCTURE: generate the flow-past-a-sphere case file
(ls-stag-3d_parallel_b200/cases/flow_sphere_128x64x64.npz) from the
reference's own mesh build and equation set-up (oracle/_ref/ref_harness,
built by oracle/build_ref.sh).  Run from the repository root:

    python oracle/make_flow_case.py

Domain [0,8] x [0,4] x [0,4] on a uniform 128 x 64 x 64 staggered grid
(h = 1/16), a sphere of diameter 1 centred at (2, 2 + h/2, 2 + h/2) (the
reference's own half-cell shift of the sphere centre,
flow_sphere_task_description.h:105-110), Re = 100, uniform inflow U = 1, the
flow task's walls and convective outflow, dt = 0.01.  Every mesh array the
GPU time step reads and the initial state are stored sparsely (the most
frequent value of each array and the exceptions), which keeps the file
small; lsstag_b200.cases.load_flow_case expands it.

The loads inputs of the same mesh (LoadsCalculator's cut-cell list,
delta_ib_max, inv_delta_ib_ne, inv_delta_ib_tn and fcoef, from the harness's
loads mode; the geometry arrays of both runs are checked equal) are stored
beside them for the drag objective of the time-step adjoint.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "ls-stag-3d_parallel_b200"))

import ref_runner as rr  # noqa: E402
from lsstag_b200 import cases  # noqa: E402

KEEP = ["dims", "celltype", "xtype", "ytype", "ztype", "side_type", "theta", "alpha", "delta", "inv_vof", "vof_x",
        "vof_y", "vof_z", "inv_mx", "inv_my", "inv_mz", "dib_en", "dib_ws", "dib_nb", "dib_st", "inv_dib_ne",
        "inv_dib_tn", "vib", "vibyx", "vibzy", "u_w", "bc", "pins", "nu_coef_coef2_integr_dt_eps_vbase_maxit",
        "restart_mom_p", "u_0", "v_0", "w_0", "p_0"]


LOADS_KEEP = ["cells", "dmax", "dne", "dtn"]


def _store(out, r, keys):
    for k in keys:
        a = np.asarray(r[k])
        if a.size < 64:
            out[k] = a
            continue
        vals, cnt = np.unique(a, return_counts=True)
        mode = vals[np.argmax(cnt)]
        idx = np.nonzero(a != mode)[0].astype(np.int64)
        out[k + "__mode"] = np.array(mode, dtype=a.dtype)
        out[k + "__idx"] = idx
        out[k + "__val"] = a[idx]
        out[k + "__n"] = np.array(a.size)


def loads_inputs(case, geom):
    """The loads inputs of the case's mesh (harness loads mode), checked
    against the flow run's geometry."""
    r = rr.run_loads(case, threads=os.cpu_count() or 1, timeout=3000)
    for k in ("celltype", "theta", "delta", "inv_vof"):
        assert np.array_equal(np.asarray(r[k]).ravel(), np.asarray(geom[k]).ravel()), k
    out = {}
    _store(out, r, LOADS_KEEP)
    out["fcoef"] = np.array(float(r["nu_fcoef_dt"][1]))
    return out


def main():
    h = 1.0 / 16
    case = rr.Case(128, 64, 64, h, h, h, spheres=[(2.0, 2.0 + 0.5 * h, 2.0 + 0.5 * h, 0.5)])
    r = rr.run(case, threads=os.cpu_count() or 1, flow_setup=1, restart=30, dump_geometry=0, timeout=3000)
    out = {}
    _store(out, r, KEEP)
    out.update(loads_inputs(case, r))
    path = cases.flow_case_path()
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
