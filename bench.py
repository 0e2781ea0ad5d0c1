#!/usr/bin/env python
"""Benchmark of the B200 pressure-Poisson projection solver.

Workload (one "step" = one complete solve from x = 0):
  standalone cut-cell pressure-Poisson system on the unit cube at 256^3 with
  four seeded immersed spheres, Neumann walls and the reference's two pinned
  rows; FGMRES(30) right-preconditioned with the reference-shaped multigrid
  (Galerkin coarse operators, ADLJ z/y/x line smoother, V(0,3)), solved to a
  relative residual of 1e-10 (absolute eps = 1e-10 * ||b||, the reference's
  stopping rule on the implicit residual).
  value     = ms per solve with the FP32 multigrid preconditioner inside FP64
              FGMRES with iterative refinement (device time, CUDA events on
              the solver's stream), inputs resident in HBM;
  fp64_ms   = the same solve with the FP64 multigrid (the plain FP64 GPU solve);
  e2e       = the FP32-preconditioned solve through the C ABI with host
              buffers (b, x in, x out, pinned host memory), copies timed;
  roofline  = the dominant kernel's algorithmic bytes / its event-timed
              duration against the measured HBM copy bandwidth;
  cpu_baseline = the reference's own MG-FGMRES (oracle/_ref, OpenMP on all
              host cores) on the same operator and right-hand side.
Multi-GPU: replicas only (each rank solves its own copy; no collectives on the
data path); the timed region is bracketed by a barrier and the max over ranks
is reported.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--size 256]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "ls-stag-3d_parallel_b200"))

METRIC = "Poisson ms/solve at 256³ to 1e-10: FP32-MG vs FP64 on 1 B200; HBM % peak"
FALLBACK_HBM_GBS = 6650.0


def measured_hbm_gbs():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [v.strip() for v in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for k, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(k)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(args, backend: str = "nccl"):
    """One process per GPU (replicas): rank/world from the torchrun
    environment; the process group only carries the barrier and the max over
    ranks of the timings (gloo on CPU for the host-side tests)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
        pg = dist
    return world, rank, local, pg


def barrier_max(pg, value: float, local: int) -> float:
    if pg is None:
        return value
    import torch
    dev = f"cuda:{local}" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


def reference_solve_ms(P, dims, b, threads, repeats):
    """Reference MG-FGMRES(30) on the host cores: per-solve seconds."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_runner as rr
    r = rr.run_planes(P, dims, b, threads=threads, fgmres=1, bicgstab=0, restart=30, rel_tol=1e-10,
                      max_it=200, repeats=repeats, timeout=3600)
    return [1e3 * t for t in r["fgmres_time_s"]], int(r["fgmres_it"][0]), int(r["omp_threads"][0]), r["fgmres_x"]


def run_reference_arm(args, world, rank):
    if rank != 0:
        return 0
    from lsstag_b200 import cases
    P, dims, pins, b = cases.load(args.size)
    threads = os.cpu_count() or 1
    cfg = config_dict(args, world)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_runner as rr
    if not rr.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_harness not built (needs the "
                          "reference sources at build time)"}))
        return 0
    warm = min(args.warmup, 1)
    times, it, th, _ = reference_solve_ms(P, dims, b, threads, warm + args.steps)
    timed = times[warm:]
    ms = sum(timed) / len(timed)
    out = {"impl": "reference", "metric": METRIC, "value": ms, "unit": "ms/solve", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
           "iterations": it,
           "cpu_baseline": {"value": ms, "unit": "ms/solve", "cores": th, "kind": "reference",
                            "sample": f"{len(timed)} full {args.size}^3 MG-FGMRES(30) solves to 1e-10 "
                                      f"(reference LS-STAG-3D OpenMP build, g++ -O2, {th} threads)"},
           "gram_schmidt": "modified Gram-Schmidt, one pass per basis vector (the reference's own)",
           "e2e": {"value": ms, "unit": "ms/solve", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))
    return 0


FLOW_METRIC = "Flow past a sphere 128x64x64 FP64 (C0): ms per time step on 1 B200"


def reference_flow_steps(steps, threads):
    """The reference's own time step (oracle/_ref, TimeSteppingMethodInterface::
    step order) on the flow case: per-step seconds and iteration counts."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_runner as rr
    h = 1.0 / 16
    case = rr.Case(128, 64, 64, h, h, h, spheres=[(2.0, 2.0 + 0.5 * h, 2.0 + 0.5 * h, 0.5)])
    r = rr.run(case, threads=threads, flow_steps=steps, flow_no_dump=1, restart=30, dump_geometry=0, timeout=3600)
    return [1e3 * t for t in r["step_s"]], [r[f"its_{k}"].tolist() for k in range(1, steps + 1)], int(r["omp_threads"][0])


def run_flow(args, world, rank, local, pg):
    """One step = one time step of the flow past a sphere (momentum equations,
    pressure equation, projection) with every operator on the GPU."""
    import torch

    from lsstag_b200 import cases
    from lsstag_b200.flow import FlowStepper, FlowStepperNative
    cfg = {"workload": "flow_sphere_128x64x64_fp64_dt0.01_Re100", "grid": [128, 64, 64],
           "bodies": "sphere D=1 at (2, 2+h/2, 2+h/2) in [0,8]x[0,4]x[0,4]",
           "solvers": "momentum ILU(0)-FGMRES(13), pressure MG-FGMRES(30), absolute eps 1e-5 (reference defaults)",
           "l2": "state and operators larger than L2", "parallelism": "replicas" if world > 1 else "single GPU"}
    if args.impl == "reference":
        if rank != 0:
            return 0
        threads = os.cpu_count() or 1
        ms, its, th = reference_flow_steps(args.warmup + args.steps, threads)
        timed = ms[args.warmup:] if len(ms) > args.warmup else ms
        v = sum(timed) / len(timed)
        print(json.dumps({"impl": "reference", "metric": FLOW_METRIC, "value": v, "unit": "ms/step", "n_gpus": world,
                          "steps": args.steps, "warmup": args.warmup, "ms_per_step": v, "higher_is_better": False,
                          "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                          "config": cfg, "iterations_last": its[-1],
                          "cpu_baseline": {"value": v, "unit": "ms/step", "cores": th, "kind": "reference",
                                           "sample": f"{len(timed)} time steps after {args.warmup}"},
                          "e2e": {"value": v, "unit": "ms/step", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return 0
    torch.cuda.set_device(local)
    g, dims, par, (u0, v0, w0, p0) = cases.load_flow_case()
    def timed(fp32, p_rel_tol=None):
        fs = FlowStepperNative(g, dims, par, u0, v0, w0, p0, device=local, pressure_mg_fp32=fp32, p_rel_tol=p_rel_tol)
        for _ in range(args.warmup):
            fs.step()
        barrier(pg)
        torch.cuda.synchronize()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record()
        its = [fs.step() for _ in range(args.steps)]
        t1.record()
        torch.cuda.synchronize()
        ms = barrier_max(pg, t0.elapsed_time(t1), local) / args.steps
        (u, v, w), p = fs.state()
        fs.close()
        return ms, its, (u, v, w, p)
    ms, its, st64 = timed(False)
    # the FP32 cycle inside FP64 FGMRES for the pressure (operator with negated pins)
    ms32, its32, st32 = timed(True)
    # the C0 specification's pressure tolerance: each solve to 1e-8 of its right-hand side
    ms_rel, its_rel, _ = timed(False, 1e-8)
    ms_rel32, its_rel32, _ = timed(True, 1e-8)
    import numpy as np
    dv = max(float(np.linalg.norm(a - b) / np.linalg.norm(b)) for a, b in zip(st32[:3], st64[:3]))
    # end to end through the host-array entry points (every vector copied in and out)
    fh = FlowStepper(g, dims, par, u0, v0, w0, p0, device=local)
    fh.step()
    torch.cuda.synchronize()
    t = time.perf_counter()
    for _ in range(args.steps):
        fh.step()
    e2e = barrier_max(pg, 1e3 * (time.perf_counter() - t), local) / args.steps
    fh.close()
    out = {"metric": FLOW_METRIC, "value": ms, "unit": "ms/step", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg, "iterations_last": its[-1],
           "driver": "native C++ time step (lsg_flow_step; momentum solves on library threads)",
           "fp32_mg_pressure": {"ms_per_step": ms32, "iterations_last": its32[-1],
                                "max_rel_velocity_diff_vs_fp64": dv,
                                "note": "pressure MG cycle in FP32 on the operator with negated pins"},
           "pressure_rel_1e-8": {"fp64_ms_per_step": ms_rel, "fp64_iterations_last": its_rel[-1],
                                 "fp32_mg_ms_per_step": ms_rel32, "fp32_mg_iterations_last": its_rel32[-1],
                                 "note": "each pressure solve to 1e-8 of its right-hand side's norm"},
           "e2e": {"value": e2e, "unit": "ms/step", "note": "host-array entry points, every operand copied"}}
    if rank == 0 and not args.no_cpu_baseline:
        try:
            ref_ms, ref_its, th = reference_flow_steps(3, os.cpu_count() or 1)
            out["cpu_baseline"] = {"value": sum(ref_ms[1:]) / 2, "unit": "ms/step", "cores": th, "kind": "reference",
                                   "iterations_last": ref_its[-1],
                                   "sample": "time steps 2-3 of the same case (reference OpenMP build)"}
        except Exception as e:  # report, do not hide
            out["cpu_baseline"] = {"error": str(e)}
    if rank == 0:
        print(json.dumps(out))
    return 0


LARGE_METRIC = "Large flow 512x256x256, 3 ellipsoids (C4), FP32-MG pressure to 1e-9: ms per time step on 1 B200"


def run_flow_large(args, world, rank, local, pg):
    """One step = one time step of the large flow: domain [0,16]x[0,8]x[0,8]
    on a uniform 512x256x256 grid (h = 1/32), three seeded ellipsoids
    (semi-axes U[0.3, 0.8], random rotations, centres in the first third),
    Re 300, dt 0.005; momentum ILU(0)-FGMRES(13) to the reference's absolute
    1e-5, pressure FGMRES(30) with the FP32 multigrid to 1e-9 relative to
    each right-hand side.  The mesh (level set to immersed-boundary
    distances) is built on the GPU from the ellipsoids; the same steps with
    the FP64 multigrid give the plain FP64 time and the state difference."""
    import numpy as np
    import torch

    from lsstag_b200 import cases, synth
    from lsstag_b200.flow import FlowStepperNative
    dims = (512, 256, 256)
    h = 1.0 / 32
    ell = synth.ellipsoids(11, 3, (16.0, 8.0, 8.0), amin=0.3, amax=0.8)
    cfg = {"workload": "flow_3ellipsoids_512x256x256_Re300_dt0.005", "grid": list(dims),
           "bodies": "3 ellipsoids, semi-axes U[0.3,0.8], random rotations, centres in the first third (seed 11)",
           "solvers": "momentum ILU(0)-FGMRES(13) absolute 1e-5; pressure FGMRES(30), FP32 multigrid, 1e-9 relative",
           "l2": "state and operators larger than L2", "parallelism": "replicas" if world > 1 else "single GPU"}
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps({"impl": "reference", "metric": LARGE_METRIC, "unavailable":
                              "the reference's CPU mesh build and time steps at 33.5M cells do not fit the bench's "
                              "time bound; its per-step cost is the 128x64x64 flow workload's reference arm"}))
        return 0
    torch.cuda.set_device(local)
    t0 = time.perf_counter()
    g, dims, par, st = cases.flow_case_on_device(dims, (h, h, h), ellipsoids=ell, Re=300.0, dt=0.005, device=local)
    setup_s = time.perf_counter() - t0
    res = {}
    for name, fp32 in (("fp32", True), ("fp64", False)):
        t1 = time.perf_counter()
        fs = FlowStepperNative(g, dims, par, *st, device=local, pressure_mg_fp32=fp32, p_rel_tol=1e-9)
        init_s = time.perf_counter() - t1
        for _ in range(args.warmup):
            fs.step()
        barrier(pg)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        its = [fs.step() for _ in range(args.steps)]
        e1.record()
        torch.cuda.synchronize()
        ms = barrier_max(pg, e0.elapsed_time(e1), local) / args.steps
        (u, v, w), p = fs.state()
        res[name] = {"ms_per_step": ms, "iterations_last": its[-1], "pressure_iterations": [i[3] for i in its],
                     "operators_setup_s": init_s, "state": (u, v, w)}
        fs.close()
        torch.cuda.empty_cache()
    dv = max(float(np.linalg.norm(a - b) / np.linalg.norm(b)) for a, b in zip(res["fp32"]["state"], res["fp64"]["state"]))
    v = res["fp32"]["ms_per_step"]
    out = {"metric": LARGE_METRIC, "value": v, "unit": "ms/step", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": v, "higher_is_better": False, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32 (multigrid) / f64", "data": "synthetic", "config": cfg,
           "fp64_ms_per_step": res["fp64"]["ms_per_step"],
           "speedup_fp32mg_vs_fp64": res["fp64"]["ms_per_step"] / v,
           "iterations_last": {k: res[k]["iterations_last"] for k in res},
           "pressure_iterations": {k: res[k]["pressure_iterations"] for k in res},
           "max_rel_velocity_diff_fp32_vs_fp64": dv,
           "mesh_and_case_setup_s": setup_s, "operators_setup_s": {k: res[k]["operators_setup_s"] for k in res},
           "cut_cells": int(g["cells"].size),
           "e2e": None, "e2e_note": "no host-array arm at this size: state and mesh are built and stay on the device"}
    if rank == 0:
        print(json.dumps(out))
    return 0


ADJ_METRIC = "Drag gradient through 50 time steps of the 128x64x64 sphere flow (C3): ms per gradient on 1 B200"


def run_adjoint(args, world, rank, local, pg):
    """One step = one gradient of the mean drag coefficient over
    --adjoint-steps time steps of the flow case (8 inflow modes and a forcing
    field), checkpoints every --checkpoint-every steps: forward, one recompute
    per segment and the reverse sweep, every operator and transposed
    operator on the GPU; --adjoint-sweep device keeps the state, the
    checkpoints and the cotangents in device memory, host runs the sweep
    through the host-array entry points."""
    import numpy as np
    import torch

    cfg = {"workload": f"adjoint_flow_sphere_128x64x64_{args.adjoint_steps}steps_ckpt{args.checkpoint_every}",
           "grid": [128, 64, 64], "objective": "mean C_d over the steps (LoadsCalculator, unfiltered)",
           "parameters": "8 inflow modes N(0,0.05) and a forcing field N(0,0.01), seed 7",
           "solvers": "forward and transposed: momentum ILU(0)-FGMRES(13), pressure MG-FGMRES(30), "
                      "absolute eps 1e-5 (reference defaults)",
           "warmup": "gradients over 1 time step (contexts, graphs and transposed operators built)",
           "sweep": args.adjoint_sweep,
           "parallelism": "replicas" if world > 1 else "single GPU"}
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps({"impl": "reference", "metric": ADJ_METRIC,
                              "unavailable": "the reference has no adjoint (its forward time step is the flow "
                                             "workload's reference arm)"}))
        return 0
    torch.cuda.set_device(local)
    from lsstag_b200 import cases
    from lsstag_b200 import flow_adjoint as FA
    g, dims, par, (u0, v0, w0, p0) = cases.load_flow_case()
    par = dict(par, fcoef=float(g["fcoef"]))
    ops = FA.GpuFlowOps(g, dims, par, device=local)
    rng = np.random.default_rng(7)
    theta = 0.05 * rng.standard_normal(8)
    forcing = [0.01 * rng.standard_normal(a.size) for a in (u0, v0, w0)]
    sweep = FA.FlowAdjointDevice if args.adjoint_sweep == "device" else FA.FlowAdjoint
    for _ in range(args.warmup):
        sweep(ops, 1, every=1).gradient(theta, forcing, (u0, v0, w0), p0)
    sweep = FA.FlowAdjointDevice if args.adjoint_sweep == "device" else FA.FlowAdjoint
    fa = sweep(ops, args.adjoint_steps, every=args.checkpoint_every)
    barrier(pg)
    torch.cuda.synchronize()
    t = time.perf_counter()
    for _ in range(args.steps):
        J, gth, gf = fa.gradient(theta, forcing, (u0, v0, w0), p0)
    torch.cuda.synchronize()
    ms = barrier_max(pg, 1e3 * (time.perf_counter() - t), local) / args.steps
    ops.close()
    out = {"metric": ADJ_METRIC, "value": ms, "unit": "ms/gradient", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg, "J": J,
           "dJ_dtheta": [float(v) for v in gth], "dJ_df_norm": float(np.sqrt(sum(a @ a for a in gf))),
           "sweep_stats": fa.stats,
           "e2e": {"value": ms, "unit": "ms/gradient", "note": "the timed value includes the upload of the "
                   "initial state and parameters and the download of the gradient"}}
    if rank == 0 and not args.no_cpu_baseline:
        try:
            ref_ms, _, th = reference_flow_steps(3, os.cpu_count() or 1)
            out["cpu_baseline"] = {"value": args.adjoint_steps * sum(ref_ms[1:]) / 2,
                                   "unit": f"ms per {args.adjoint_steps} forward time steps", "cores": th,
                                   "kind": "reference",
                                   "sample": "time steps 2-3 of the same case, scaled to the step count: the "
                                             "reference has no adjoint, this is its forward cost alone"}
        except Exception as e:  # report, do not hide
            out["cpu_baseline"] = {"error": str(e)}
    if rank == 0:
        print(json.dumps(out))
    return 0


def config_dict(args, world):
    return {"workload": f"poisson_spheres4_{args.size}^3_mgfgmres30_rel1e-10",
            "grid": [args.size] * 3, "bodies": "4 seeded spheres (seed 3), Neumann walls, 2 pinned rows",
            "krylov": f"FGMRES({getattr(args, 'restart', 30)}) FP64, modified Gram-Schmidt projections",
            "precond": ("Galerkin MG, red-black / 8-colour Gauss-Seidel V(2,2)"
                        if getattr(args, "smoother", "adlj") == "rbgs"
                        else "Galerkin MG, ADLJ z/y/x line smoother V(0,3), omega 0.805"),
            "l2": "inputs larger than L2 (operator 0.94 GB FP64 + Krylov basis)",
            "pins": getattr(args, "pins", "reference"),
            "parallelism": "replicas" if world > 1 else "single GPU"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--size", type=int, default=256)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--restart", type=int, default=30, help="FGMRES restart length (30 = the measured workload)")
    ap.add_argument("--smoother", default="adlj", choices=["adlj", "rbgs"],
                    help="multigrid smoother of both arms: the reference's ADLJ V(0,3) (default) or the "
                         "red-black Gauss-Seidel V(2,2) variant")
    ap.add_argument("--gs", default="lowsync", choices=["mgs", "lowsync"],
                    help="Gram-Schmidt form of both arms: the low-synchronisation form of the MGS "
                         "projections (default; two passes over the basis per step) or the reference's "
                         "pass-per-vector MGS")
    ap.add_argument("--workload", default="poisson", choices=["poisson", "flow", "adjoint", "flow_large"],
                    help="poisson: the 256^3 pressure solve (the headline); flow: time steps of the flow past "
                         "a sphere at 128x64x64 (every operator of the step on the GPU); adjoint: the drag "
                         "gradient through time steps of that flow (use --steps 1)")
    ap.add_argument("--pins", default="reference", choices=["reference", "negated"],
                    help="poisson workload, this arm: the reference's +1 identity pins (default) or the same "
                         "system with the pinned rows negated")
    ap.add_argument("--adjoint-steps", type=int, default=50, help="time steps of one adjoint gradient")
    ap.add_argument("--checkpoint-every", type=int, default=10, help="checkpoint interval of the adjoint sweep")
    ap.add_argument("--adjoint-sweep", default="device", choices=["device", "host"],
                    help="device: state and cotangents in device memory (FlowAdjointDevice); host: the sweep over "
                         "the host-array entry points (FlowAdjoint)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "b200" else args.warmup
    world, rank, local, pg = dist_setup(args)
    if args.workload in ("flow", "adjoint", "flow_large"):
        rc = {"flow": run_flow, "adjoint": run_adjoint, "flow_large": run_flow_large}[args.workload](
            args, world, rank, local, pg)
        if pg is not None:
            pg.destroy_process_group()
        return rc
    if args.impl == "reference":
        rc = run_reference_arm(args, world, rank)
        if pg is not None:
            pg.destroy_process_group()
        return rc

    import numpy as np
    import torch

    from lsstag_b200 import _lib as L
    from lsstag_b200 import cases
    from lsstag_b200 import solver as S

    torch.cuda.set_device(local)
    # the operator as the product builds it: the flow task's mesh build and
    # the Laplace assembly on the GPU from the seeded spheres alone; where a
    # case file holds the reference's own assembly of the same case, the two
    # must be equal bit for bit
    t0 = time.perf_counter()
    P, dims, pins, b, mesh_ms = cases.build_on_device(args.size, 3, device=local)
    setup_wall_ms = 1e3 * (time.perf_counter() - t0)
    operator_bitwise = None
    if os.path.isfile(cases.case_path(args.size)):
        P_ref, _, pins_ref, b_ref = cases.load(args.size)
        operator_bitwise = bool(P_ref.tobytes() == P.tobytes() and np.array_equal(pins_ref, pins)
                                and np.array_equal(b_ref, b))
        del P_ref, b_ref
    if args.pins == "negated":
        # the same system with the pinned rows negated (b is 0 there: same
        # solution); the multigrid hierarchy then has no wrong-signed rows
        P = S.pins_negated(P, pins)
    n = b.size
    bnorm = float(np.linalg.norm(b))
    task = S.Task(eps=1e-10 * bnorm, MAX_ITER=200, FGMRES_RESTART_NUM=args.restart,
                  n_post=2 if args.smoother == "rbgs" else 3)
    dev = f"cuda:{local}"
    b_dev = torch.from_numpy(b).to(dev)
    results = {}
    gs = L.GS_LOWSYNC if args.gs == "lowsync" else L.GS_MGS
    for name, prec in (("fp32", L.FP32), ("fp64", L.FP64)):
        if args.smoother == "rbgs":
            s = S.MGFGMRES(device=local, mg_precision=prec, gram_schmidt=gs, smoother=L.SMOOTHER_RBGS, n_pre=2)
        else:
            s = S.MGFGMRES(device=local, mg_precision=prec, gram_schmidt=gs)
        s.set_planes(P, dims, task)
        setup_ms = s.setup_times()
        x_dev = torch.zeros(n, dtype=torch.float64, device=dev)
        st = L.Stats()
        def one():
            x_dev.zero_()
            torch.cuda.synchronize()
            s.ctx.check(s.ctx.lib.lsg_solve_device(s.ctx.h, L.C.c_void_p(b_dev.data_ptr()),
                                                   L.C.c_void_p(x_dev.data_ptr()), L.C.byref(st)))
            return st.ms, st.iterations, st.kernel_launches, st.bytes, st.true_residual, st.norm_r
        for _ in range(args.warmup):
            one()
        barrier(pg)
        torch.cuda.synchronize()
        sampler = ClockSampler(local) if name == "fp32" else None
        if sampler:
            sampler.__enter__()
        torch.cuda.nvtx.range_push(f"lsg_{name}_timed")   # ncu --nvtx-include lsg_fp32_timed/
        recs = [one() for _ in range(args.steps)]
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        if sampler:
            sampler.__exit__()
        barrier(pg)
        ms = sum(r[0] for r in recs)
        ms_max = barrier_max(pg, ms, local)
        results[name] = {"ms_total": ms_max, "ms_per_solve": ms_max / args.steps, "it": recs[-1][1],
                         "launches": sum(r[2] for r in recs), "bytes": recs[-1][3], "true_res": recs[-1][4],
                         "norm_r": recs[-1][5], "x": x_dev.cpu().numpy(), "clocks": sampler.summary() if sampler else None,
                         "setup": {"operator_and_row_dictionary_ms": setup_ms[0], "hierarchy_ms": setup_ms[1]}}
        if name == "fp32":
            # dominant-kernel roofline (finest-level smoother/residual kernels)
            prof = {}
            nv = recs[-1][1]
            per_solve = {0: 3 * nv, 1: 3 * nv, 2: 3 * nv, 3: 9 * nv, 5: 9 * nv, 9: 3 * nv, 10: 3 * nv, 11: 3 * nv}
            names = {0: "adlj_xline_fp32", 1: "adlj_yline_fp32", 2: "adlj_zline_fp32", 3: "residual7_fp32",
                     5: "residual27_level1_fp32", 9: "adlj_fused_x_fp32", 10: "adlj_fused_y_fp32",
                     11: "adlj_fused_z_fp32"}
            # the finest level runs the fused direction steps (ids 9-11) unless
            # its shape needs the separate residual and line-solve kernels
            msk, byk = L.C.c_double(0), L.C.c_double(0)
            fused = s.ctx.lib.lsg_profile_kernel(s.ctx.h, 9, 1, L.C.byref(msk), L.C.byref(byk)) == L.LSG_OK
            for k in ((9, 10, 11, 5) if fused else (0, 1, 2, 3, 5)):
                msk = L.C.c_double(0)
                byk = L.C.c_double(0)
                s.ctx.check(s.ctx.lib.lsg_profile_kernel(s.ctx.h, k, 20, L.C.byref(msk), L.C.byref(byk)))
                prof[k] = (msk.value, byk.value, per_solve[k] * msk.value)
            results["prof"] = {names[k]: {"ms": v[0], "bytes": v[1], "gbs": v[1] / v[0] / 1e6, "ms_per_solve": v[2]}
                               for k, v in prof.items()}
            kdom = max(prof, key=lambda k: prof[k][2])
            results["dominant"] = (names[kdom], prof[kdom])
            # e2e through the C ABI with pinned host buffers
            bh = torch.from_numpy(b).pin_memory()
            xh = torch.zeros(n, dtype=torch.float64).pin_memory()
            e2e = []
            for rep in range(args.warmup + args.steps):
                xh.zero_()
                t0 = time.perf_counter()
                s.ctx.check(s.ctx.lib.lsg_solve(s.ctx.h, L.C.cast(bh.data_ptr(), L.C.POINTER(L.C.c_double)),
                                                L.C.cast(xh.data_ptr(), L.C.POINTER(L.C.c_double)), L.C.byref(st)))
                if rep >= args.warmup:
                    e2e.append(1e3 * (time.perf_counter() - t0))
            results["e2e_ms"] = barrier_max(pg, sum(e2e), local) / args.steps
        s.close()
        del x_dev
    # the mixed-precision configuration's point smoother: red-black / 8-colour
    # Gauss-Seidel V(2,2) with the FP32 cycle, same operator and tolerance
    rb = None
    if args.smoother == "adlj":
        s = S.MGFGMRES(device=local, mg_precision=L.FP32, gram_schmidt=gs, smoother=L.SMOOTHER_RBGS, n_pre=2)
        s.set_planes(P, dims, S.Task(eps=1e-10 * bnorm, MAX_ITER=200, FGMRES_RESTART_NUM=args.restart, n_post=2))
        x_dev = torch.zeros(n, dtype=torch.float64, device=dev)
        st = L.Stats()
        rms = []
        for rep in range(2 + 3):
            x_dev.zero_()
            torch.cuda.synchronize()
            s.ctx.check(s.ctx.lib.lsg_solve_device(s.ctx.h, L.C.c_void_p(b_dev.data_ptr()),
                                                   L.C.c_void_p(x_dev.data_ptr()), L.C.byref(st)))
            if rep >= 2:
                rms.append(st.ms)
        rb = {"ms_per_solve": barrier_max(pg, sum(rms), local) / len(rms), "iterations": st.iterations,
              "true_rel_residual": st.true_residual / bnorm, "solves_timed": len(rms),
              "smoother": "red-black (7-point level) / 8-colour (27-point levels) Gauss-Seidel V(2,2), FP32 cycle"}
        s.close()
        del x_dev
    # the FP64 cycle with the fused direction steps asked for explicitly (the
    # default FP64 cycle keeps the reference's schedule)
    fp64_fused = None
    if args.smoother == "adlj":
        s = S.MGFGMRES(device=local, mg_precision=L.FP64, gram_schmidt=gs, adlj_schedule=L.ADLJ_FUSED)
        s.set_planes(P, dims, task)
        x_dev = torch.zeros(n, dtype=torch.float64, device=dev)
        st = L.Stats()
        recs = []
        for k in range(args.warmup + args.steps):
            x_dev.zero_()
            torch.cuda.synchronize()
            s.ctx.check(s.ctx.lib.lsg_solve_device(s.ctx.h, L.C.c_void_p(b_dev.data_ptr()),
                                                   L.C.c_void_p(x_dev.data_ptr()), L.C.byref(st)))
            if k >= args.warmup:
                recs.append((st.ms, st.iterations))
        xf = x_dev.cpu().numpy()
        ms_f = barrier_max(pg, sum(r[0] for r in recs), local) / args.steps
        fp64_fused = {"ms_per_solve": ms_f, "iterations": recs[-1][1],
                      "rel_l2_vs_fp64": float(np.linalg.norm(xf - results["fp64"]["x"]) /
                                              np.linalg.norm(results["fp64"]["x"])),
                      "note": "FP64 cycle with LSG_ADLJ_FUSED (the default FP64 cycle keeps the reference's "
                              "r -= A c, line solve schedule)"}
        s.close()
        del x_dev
    x32, x64 = results["fp32"]["x"], results["fp64"]["x"]
    err = float(np.linalg.norm(x32 - x64) / np.linalg.norm(x64))
    peak, peak_kind = measured_hbm_gbs()
    dname, (dms, dbytes, _) = results["dominant"]
    achieved = dbytes / dms / 1e6
    traffic = None
    tp = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.isfile(tp):
        try:
            with open(tp) as f:
                tj = json.load(f)
            traffic = tj.get(dname, {}).get(f"traffic_bytes_per_launch_{args.size}")
        except Exception:
            traffic = None
    value = results["fp32"]["ms_total"] / (args.steps * world)
    out = {
        "metric": METRIC, "value": value, "unit": "ms/solve", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": results["fp32"]["ms_per_solve"], "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (multigrid) / f64 (Krylov)", "data": "synthetic",
        "config": config_dict(args, world),
        "fp64_ms_per_solve": results["fp64"]["ms_per_solve"],
        "fp64_fused_schedule": fp64_fused,
        "speedup_fp32mg_vs_fp64": results["fp64"]["ms_per_solve"] / results["fp32"]["ms_per_solve"],
        "iterations": {"fp32": results["fp32"]["it"], "fp64": results["fp64"]["it"]},
        "true_rel_residual": {"fp32": results["fp32"]["true_res"] / bnorm, "fp64": results["fp64"]["true_res"] / bnorm},
        "rel_l2_fp32_vs_fp64": err,
        "gram_schmidt": f"modified Gram-Schmidt, {args.gs} schedule",
        "operator": {"built_on_gpu_from_seed": True, "bitwise_equal_to_reference_assembly": operator_bitwise,
                     "mesh_build_ms": mesh_ms, "case_build_wall_ms": setup_wall_ms},
        "solve_algorithmic_gbs": results["fp32"]["bytes"] / results["fp32"]["ms_per_solve"] / 1e6,
        "roofline": {"bound": "hbm", "kernel": dname, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic,
                     "algorithmic_bytes_per_launch": dbytes, "ms_per_launch": dms},
        "kernels": results["prof"],
        "setup_ms": {k: results[k]["setup"] for k in ("fp32", "fp64")},
        "rbgs_v22_fp32": rb,
        "adlj_schedule": {"fp32": "fused direction steps on the finest level (residual formed in the line solve)"
                          if any(k.startswith("adlj_fused") for k in results["prof"]) else
                          "reference schedule (r -= A c, then the line solve)",
                          "fp64": "reference schedule (r -= A c, then the line solve)"},
        "e2e": {"value": results["e2e_ms"] / world, "unit": "ms/solve", "h2d_bytes_per_step": 2 * 8 * n,
                "d2h_bytes_per_step": 8 * n},
        "gpu_launches": results["fp32"]["launches"],
        "clocks": results["fp32"]["clocks"],
    }
    if rank == 0 and not args.no_cpu_baseline:
        try:
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            import ref_runner as rr
            if rr.available():
                threads = os.cpu_count() or 1
                times, it, th, x_ref = reference_solve_ms(P, dims, b, threads, 1)
                out["cpu_baseline"] = {"value": times[0], "unit": "ms/solve", "cores": th, "kind": "reference",
                                       "iterations": it,
                                       "sample": f"one full {args.size}^3 MG-FGMRES(30) solve to 1e-10 on the same "
                                                 f"operator and right-hand side (reference OpenMP build, g++ -O2, "
                                                 f"{th} threads)"}
                rn = float(np.linalg.norm(x_ref))
                out["rel_l2_vs_reference"] = {"fp32": float(np.linalg.norm(x32 - x_ref) / rn),
                                              "fp64": float(np.linalg.norm(x64 - x_ref) / rn),
                                              "reference_iterations": it}
            else:
                out["cpu_baseline"] = None
        except Exception as e:  # report, do not hide
            out["cpu_baseline"] = {"error": str(e)}
    if rank == 0:
        print(json.dumps(out))
    if pg is not None:
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
