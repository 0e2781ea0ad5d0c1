"""TEST INFRASTRUCTURE: run the reference-backed harness binary
(``oracle/_ref/ref_harness``, built by ``oracle/build_ref.sh`` from the
reference's own sources) and load what it dumps.

Only tests, the fixture generator and bench.py's CPU-baseline leg use this
module; the product never does.
"""
from __future__ import annotations

import os
import subprocess
import tempfile
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_BIN = os.path.join(HERE, "_ref", "ref_harness")
# the same harness built with the reference's pressure solver swapped for the
# B200 library through include/lsstag_b200_adapter.hpp (-DLS_STAG_USE_B200)
DROPIN_BIN = os.path.join(HERE, "_ref", "ref_harness_b200")


def available(binary: str = REF_BIN) -> bool:
    return os.path.isfile(binary) and os.access(binary, os.X_OK)


@dataclass
class Case:
    """Uniform box [0, N*hx] x [0, M*hy] x [0, K*hz] with level-set bodies."""
    N: int
    M: int
    K: int
    hx: float
    hy: float
    hz: float
    spheres: list = field(default_factory=list)      # (cx, cy, cz, r)
    ellipsoids: list = field(default_factory=list)   # (c[3], axes[3], rot[3x3])

    def config_lines(self):
        lines = [f"N {self.N}", f"M {self.M}", f"K {self.K}",
                 f"hx {self.hx!r}", f"hy {self.hy!r}", f"hz {self.hz!r}"]
        for (cx, cy, cz, r) in self.spheres:
            lines.append(f"body 0 {cx!r} {cy!r} {cz!r} {r!r}")
        for (c, ax, rot) in self.ellipsoids:
            rr = " ".join(repr(float(v)) for v in np.asarray(rot).reshape(-1))
            lines.append(f"body 1 {float(c[0])!r} {float(c[1])!r} {float(c[2])!r} "
                         f"{float(ax[0])!r} {float(ax[1])!r} {float(ax[2])!r} {rr}")
        return lines


def load_dir(d: str) -> dict:
    out = {}
    with open(os.path.join(d, "manifest.txt")) as f:
        for line in f:
            name, dt, n = line.split()
            out[name] = np.fromfile(os.path.join(d, name + ".bin"), dtype=np.dtype(dt), count=int(n))
    return out


def run(case: Case, rhs: np.ndarray | None = None, *, threads: int = 0, workdir: str | None = None,
        timeout: float = 3600, binary: str = REF_BIN, **opts) -> dict:
    """Run the harness once.  ``opts`` become config keys (restart, max_it,
    rel_tol, abs_tol, fgmres, bicgstab, dump_mg, dump_geometry, dump_matrix,
    repeats, n_post).  ``binary`` = DROPIN_BIN runs the drop-in build."""
    if not available(binary):
        raise FileNotFoundError(binary)
    own = workdir is None
    d = tempfile.mkdtemp(prefix="lsg_ref_") if own else workdir
    os.makedirs(d, exist_ok=True)
    lines = case.config_lines()
    if threads:
        lines.append(f"threads {threads}")
    for k, v in opts.items():
        lines.append(f"{k} {v!r}" if isinstance(v, float) else f"{k} {v}")
    if rhs is not None:
        p = os.path.join(d, "rhs.in")
        np.ascontiguousarray(rhs, dtype=np.float64).tofile(p)
        lines.append(f"rhs {p}")
    cfg = os.path.join(d, "case.cfg")
    with open(cfg, "w") as f:
        f.write("\n".join(lines) + "\n")
    subprocess.run([binary, cfg, d], check=True, timeout=timeout,
                   stdout=subprocess.DEVNULL, stderr=subprocess.PIPE)
    res = load_dir(d)
    if own:
        import shutil
        shutil.rmtree(d, ignore_errors=True)
    return res


def csr(res: dict, name: str):
    """(rowptr, col, val, (N, M, K)) of a dumped CSR matrix."""
    dims = res[name + "_dims"]
    return (res[name + "_rowptr"], res[name + "_col"], res[name + "_val"],
            (int(dims[0]), int(dims[1]), int(dims[2])))


def run_planes(planes: np.ndarray, dims, rhs: np.ndarray, *, threads: int = 0, timeout: float = 3600,
               **opts) -> dict:
    """Reference MG-FGMRES / ILU-BiCGStab (opts fgmres=1, bicgstab=0/1) on an
    operator given as seven coefficient planes (b, s, w, p, e, n, t)."""
    if not available():
        raise FileNotFoundError(REF_BIN)
    import shutil
    d = tempfile.mkdtemp(prefix="lsg_refp_")
    try:
        pp = os.path.join(d, "planes.in")
        bp = os.path.join(d, "rhs.in")
        np.ascontiguousarray(planes, dtype=np.float64).tofile(pp)
        np.ascontiguousarray(rhs, dtype=np.float64).tofile(bp)
        N, M, K = dims
        lines = [f"N {N}", f"M {M}", f"K {K}", f"planes_in {pp}", f"rhs {bp}"]
        if threads:
            lines.append(f"threads {threads}")
        for k, v in opts.items():
            lines.append(f"{k} {v!r}" if isinstance(v, float) else f"{k} {v}")
        cfg = os.path.join(d, "case.cfg")
        with open(cfg, "w") as f:
            f.write("\n".join(lines) + "\n")
        subprocess.run([REF_BIN, cfg, d], check=True, timeout=timeout, stdout=subprocess.DEVNULL,
                       stderr=subprocess.PIPE)
        return load_dir(d)
    finally:
        shutil.rmtree(d, ignore_errors=True)


def csr_to_planes(rowptr, col, val, dims) -> np.ndarray:
    """Seven coefficient planes (b, s, w, p, e, n, t) of a 7-point CSR."""
    N, M, K = dims
    n = N * M * K
    NM = N * M
    rows = np.repeat(np.arange(n), np.diff(rowptr))
    dlt = col.astype(np.int64) - rows
    slot = np.select([dlt == -NM, dlt == -N, dlt == -1, dlt == 0, dlt == 1, dlt == N, dlt == NM],
                     [0, 1, 2, 3, 4, 5, 6], -1)
    if np.any(slot < 0):
        raise ValueError("not a 7-point operator")
    P = np.zeros((7, n))
    P[slot, rows] = val          # assignment keeps the sign of a stored -0.0
    return P


def run_projection(case: Case, u: np.ndarray, v: np.ndarray, w: np.ndarray, p: np.ndarray, abs_tol: float, *,
                   threads: int = 1, timeout: float = 3600, **opts) -> dict:
    """One pressure projection of the reference's time step on given predicted
    velocities u (x-grid), v (y-grid), w (z-grid) and pressure p: right-hand
    side, MG-FGMRES pressure correction to the absolute tolerance abs_tol, and
    the corrected u, v, w, p (harness ``projection`` mode)."""
    if not available():
        raise FileNotFoundError(REF_BIN)
    d = tempfile.mkdtemp(prefix="lsg_proj_")
    try:
        lines = case.config_lines()
        if threads:
            lines.append(f"threads {threads}")
        for k, val in opts.items():
            lines.append(f"{k} {val!r}" if isinstance(val, float) else f"{k} {val}")
        for key, arr in (("proj_u", u), ("proj_v", v), ("proj_w", w), ("proj_p", p)):
            path = os.path.join(d, key + ".in")
            np.ascontiguousarray(arr, dtype=np.float64).tofile(path)
            lines.append(f"{key} {path}")
        n = case.N * case.M * case.K
        rhs = os.path.join(d, "rhs.in")
        np.zeros(n).tofile(rhs)
        lines += [f"rhs {rhs}", f"abs_tol {float(abs_tol)!r}", "projection 1", "dump_projection 1"]
        cfg = os.path.join(d, "case.cfg")
        with open(cfg, "w") as f:
            f.write("\n".join(lines) + "\n")
        subprocess.run([REF_BIN, cfg, d], check=True, timeout=timeout, stdout=subprocess.DEVNULL,
                       stderr=subprocess.PIPE)
        return load_dir(d)
    finally:
        import shutil
        shutil.rmtree(d, ignore_errors=True)


def run_momentum(case: Case, rhs_xyz, rel_tol: float = 1e-10, *, threads: int = 1, timeout: float = 3600,
                 **opts) -> dict:
    """The reference's momentum equations for a case (harness ``momentum``
    mode): Helmholtz operators Kx/Ky/Kz and convective operators Cx/Cy/Cz in
    CSR form, and the momentum solver (ILU-FGMRES) on each K with the given
    right-hand sides (x-, y-, z-grid) to rel_tol * ||rhs||."""
    if not available():
        raise FileNotFoundError(REF_BIN)
    d = tempfile.mkdtemp(prefix="lsg_mom_")
    try:
        lines = case.config_lines()
        if threads:
            lines.append(f"threads {threads}")
        for k, val in opts.items():
            lines.append(f"{k} {val!r}" if isinstance(val, float) else f"{k} {val}")
        for name, arr in zip("xyz", rhs_xyz):
            path = os.path.join(d, f"mom_rhs_{name}.in")
            np.ascontiguousarray(arr, dtype=np.float64).tofile(path)
            lines.append(f"mom_rhs_{name} {path}")
        n = case.N * case.M * case.K
        rhs = os.path.join(d, "rhs.in")
        np.zeros(n).tofile(rhs)
        lines += [f"rhs {rhs}", "abs_tol 1.0", "momentum 1", f"mom_rel_tol {float(rel_tol)!r}"]
        cfg = os.path.join(d, "case.cfg")
        with open(cfg, "w") as f:
            f.write("\n".join(lines) + "\n")
        subprocess.run([REF_BIN, cfg, d], check=True, timeout=timeout, stdout=subprocess.DEVNULL,
                       stderr=subprocess.PIPE)
        return load_dir(d)
    finally:
        import shutil
        shutil.rmtree(d, ignore_errors=True)


def run_loads_probe(dims, inputs: dict, nu: float, *, filter_in=None, dt: float = 0.01,
                    timeout: float = 600) -> dict:
    """The reference's per-cut-cell load kernel (LoadsCalculator::calc) and
    moment kernels on given arrays.  ``inputs`` holds type (int32 n), cells
    (int32, base indices), theta, delta, vib, vibyx, vibzy, dne, dtn, dmax,
    nodes (3n each, xyz interleaved), center (3), invv, p (n), ux, uy, uz (the
    staggered grids) and optionally nucell (n).  ``filter_in`` runs the moment
    filter on a signal."""
    if not available():
        raise FileNotFoundError(REF_BIN)
    import shutil
    d = tempfile.mkdtemp(prefix="lsg_refl_")
    try:
        N, M, K = dims
        lines = [f"N {N}", f"M {M}", f"K {K}", "loads_probe 1", f"nu {nu!r}",
                 f"count {len(inputs['cells'])}", f"dt {dt!r}"]
        for k, v in inputs.items():
            p = os.path.join(d, k + ".in")
            dt_ = np.int32 if k in ("type", "cells") else np.float64
            np.ascontiguousarray(v, dtype=dt_).tofile(p)
            lines.append(f"lp_{k} {p}")
        if filter_in is not None:
            p = os.path.join(d, "filter.in")
            np.ascontiguousarray(filter_in, dtype=np.float64).tofile(p)
            lines += [f"filter_len {len(filter_in)}", f"filter_in {p}"]
        cfg = os.path.join(d, "case.cfg")
        with open(cfg, "w") as f:
            f.write("\n".join(lines) + "\n")
        subprocess.run([REF_BIN, cfg, d], check=True, timeout=timeout, stdout=subprocess.DEVNULL,
                       stderr=subprocess.PIPE)
        return load_dir(d)
    finally:
        shutil.rmtree(d, ignore_errors=True)


def run_loads(case: Case, *, threads: int = 1, timeout: float = 600, **opts) -> dict:
    """LoadsCalculator::calculate on the case's cut cells, with the seeded
    velocities, pressure and immersed-boundary velocities the harness sets."""
    return run(case, threads=threads, timeout=timeout, loads=1, dump_geometry=0, **opts)
