"""Host side of the multi-GPU bench (replicas, one process per GPU): the max
over ranks of the timings and rank 0 alone reporting, checked with two gloo
ranks on the CPU."""
import os
import socket
import subprocess
import sys
import textwrap

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = textwrap.dedent("""
    import io, contextlib, json, os, sys
    sys.path.insert(0, {root!r})
    sys.path.insert(0, os.path.join({root!r}, "ls-stag-3d_parallel_b200"))
    import bench
    world, rank, local, pg = bench.dist_setup(None, backend="gloo")
    assert world == 2 and pg is not None
    bench.barrier(pg)
    m = bench.barrier_max(pg, 1.5 + rank, local)
    out = io.StringIO()
    with contextlib.redirect_stdout(out):
        rc = bench.run_reference_arm(None, world, rank) if rank == 1 else 0
    print(json.dumps({{"rank": rank, "max": m, "rc": rc, "printed": out.getvalue()}}))
    pg.destroy_process_group()
""")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_max_and_silent_rank():
    import json
    port = _free_port()
    code = CHILD.format(root=ROOT)
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        o, e = p.communicate(timeout=120)
        assert p.returncode == 0, e
        outs.append(json.loads(o.strip().splitlines()[-1]))
    for r in outs:
        assert r["max"] == 2.5                 # max over ranks of (1.5 + rank)
    silent = [r for r in outs if r["rank"] == 1][0]
    assert silent["rc"] == 0 and silent["printed"] == ""
