"""The multi-rank path of bench.py on CPU: two gloo ranks, as torchrun starts them.

With N GPUs the benchmark runs one independent replica per rank ("replicas only": the
step has no exchange between GPUs), takes the slowest rank's time after a barrier, and
reports the whole-job rate.  These tests run that plumbing with world size 2 over gloo
on 127.0.0.1; the replica work is an oracle force evaluation on a small seeded system.
"""
import json
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import json, os, sys, time
sys.path.insert(0, {root!r})
sys.path.insert(0, os.path.join({root!r}, "oracle"))
import numpy as np
import bench
import pyoracle as po
from particlebase_b200 import workloads as W

d = bench.Dist(use_cuda=False)
s = W.fcc_system(5, 0.8442, 0.72, seed=2 + d.rank)   # this rank's replica, as bench.py seeds it
d.barrier()
t0 = time.perf_counter()
o = po.Oracle(s.box, s.lj, s.rc, s.r, types=s.types)
o.forces()
F = o.get("F")
t = time.perf_counter() - t0 + 0.05 * d.rank            # rank 1 is the slow one
d.barrier()
t_max = d.reduce(t, "max")
atoms = d.reduce(float(s.n), "sum")
print(json.dumps({{"rank": d.rank, "ws": d.ws, "t": t, "t_max": t_max, "atoms": atoms,
                  "vsum": float(np.abs(s.v).sum()), "fmax": float(np.abs(F).max()),
                  "rate": bench.replica_rate(d.ws, s.n, 1, t_max)}}))
d.close()
"""


def _free_port() -> int:
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def _run_ranks(code: str, ws: int = 2, timeout: float = 180.0):
    port = _free_port()
    procs = []
    for r in range(ws):
        env = dict(os.environ, WORLD_SIZE=str(ws), RANK=str(r), LOCAL_RANK=str(r),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env, cwd=ROOT,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    try:
        for p in procs:
            out, err = p.communicate(timeout=timeout)
            assert p.returncode == 0, err[-2000:]
            outs.append(out)
    finally:
        for p in procs:
            if p.poll() is None:
                p.kill()
    return outs


def test_two_ranks_take_the_slowest_time_and_report_the_whole_job():
    outs = _run_ranks(CHILD.format(root=ROOT))
    res = sorted((json.loads(o.strip().splitlines()[-1]) for o in outs), key=lambda r: r["rank"])
    assert [r["ws"] for r in res] == [2, 2]
    # both ranks agree on the maximum of their times, and it is the slow rank's own
    assert res[0]["t_max"] == res[1]["t_max"] == max(r["t"] for r in res)
    assert res[0]["t_max"] == res[1]["t"]
    # the whole-job rate counts both replicas against the slowest time
    n = 500
    assert res[0]["atoms"] == 2 * n
    assert res[0]["rate"] == res[1]["rate"] == 2 * n * 1 / res[0]["t_max"]
    # the replicas are independent: each rank seeds its own velocities
    assert res[0]["vsum"] != res[1]["vsum"]
    # a perfect lattice: no net force on any atom in either replica
    assert max(r["fmax"] for r in res) < 1e-9


def test_reference_arm_runs_on_rank_zero_only():
    """Under torchrun the reference arm prints from rank 0; other ranks exit 0 silently."""
    env = dict(os.environ, WORLD_SIZE="2", RANK="1", LOCAL_RANK="1")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference"],
                       env=env, cwd=ROOT, capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr[-2000:]
    assert p.stdout.strip() == ""


def test_replica_rate_is_weak_scaling():
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    one = bench.replica_rate(1, 1_048_576, 100, 0.0415)
    assert abs(bench.replica_rate(4, 1_048_576, 100, 0.0415) - 4 * one) < 1e-6 * one
