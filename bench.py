"""Benchmark of the LJ cell-list MD step on B200.

Workload (default): 1,048,576-atom Lennard-Jones fcc system (64^3 x 4),
density 0.8442, T* 0.72, rc 2.5, Gaussian isokinetic thermostat, FP32
positions/velocities/forces with FP64 reductions, dt 0.005, cell list rebuilt
every step.  Metric: atom-steps/s (N x steps / device seconds).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Timing: W untimed warm-up steps, then K timed steps in CUDA-graph units of 2
steps, each unit bracketed by CUDA events on the handle's stream with the L2
flushed (a 256 MB write) before it; value = N * K / sum of unit times, max over
ranks.  With --gpus N > 1 (torchrun) every rank runs its own replica of the
system (the path does not shard across GPUs: replicas only, weak scaling).

`e2e` runs the reference driver loop through the public API with host
buffers over the workload's 500 steps: handle set-up and import from host
memory, then per step one pb_md_run call and a temperature read-back (as
testMD2.cu:149-168 does), then the final positions copied back; wall-clock
time.  `cpu_baseline` is the FP64 oracle (OpenMP,
all host cores) on a bounded sample of the same system.  `--impl reference`
times the reference's own MD kernels compiled for the CPU (oracle/_ref), or the
oracle port where that build is absent.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

DT = 0.005
METRIC = "LJ atom-steps/s at 1M atoms (Gaussian NVT, cell list rebuilt every step)"
UNIT = "atom-steps/s"
WORKLOAD = "lj_fcc_1048576_gauss_rho0.8442_T0.72_rc2.5"
C2_STEPS = 500  # steps of the 1,048,576-atom Gaussian workload


# --------------------------------------------------------------------------- utils


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def replica_rate(ws: int, atoms: int, steps: int, seconds_max: float) -> float:
    """Whole-job atom-steps/s of `ws` independent replicas of `atoms` atoms each
    (one per rank, weak scaling), from the slowest rank's time."""
    return ws * atoms * steps / seconds_max


class Dist:
    """torch.distributed plumbing: barrier and max/sum over ranks."""

    def __init__(self, use_cuda: bool):
        self.ws, self.rank, self.local = dist_env()
        self.pg = None
        if self.ws > 1:
            import datetime
            import torch
            import torch.distributed as td
            backend = "nccl" if use_cuda else "gloo"
            td.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
            self.td, self.torch = td, torch
            self.dev = torch.device("cuda", self.local) if use_cuda else torch.device("cpu")

    def barrier(self):
        if self.ws > 1:
            self.td.barrier()

    def reduce(self, x: float, op: str) -> float:
        if self.ws == 1:
            return x
        t = self.torch.tensor([x], dtype=self.torch.float64, device=self.dev)
        self.td.all_reduce(t, op=self.td.ReduceOp.MAX if op == "max" else self.td.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.ws > 1:
            self.td.destroy_process_group()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    mx.append(float(f[2]))
                except ValueError:
                    continue
                for n, v in zip(names, f[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
        finally:
            if self.path and os.path.exists(self.path):
                os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks() -> dict:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return json.load(fh)
    except Exception:
        return {}


def profiled_traffic(name: str):
    """DRAM bytes per launch recorded from an ncu capture (profiles/*.txt)."""
    path = os.path.join(ROOT, "profiles", "traffic.txt")
    try:
        for line in open(path):
            k, _, v = line.partition(":")
            if k.strip() == name:
                return float(v.split()[0])
    except Exception:
        pass
    return None


# --------------------------------------------------------------------------- CPU arms

def run_cpu_oracle(steps: int) -> dict:
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    from particlebase_b200 import workloads as W
    po.build(ref=True)
    s = W.config_c2()
    O = po.Oracle(s.box, s.lj, s.rc, s.r, s.v)
    O.run(1, DT, mode="gauss")  # warm
    t = time.perf_counter()
    O.run(steps, DT, mode="gauss")
    el = time.perf_counter() - t
    return {"value": s.n * steps / el, "unit": UNIT, "cores": po.lib().orc_threads(),
            "kind": "port",
            "sample": f"{steps} Gaussian steps of the full 1,048,576-atom system, FP64 oracle "
                      f"(oracle/oracle.cpp), OpenMP", "seconds": el}


def run_reference_arm(args) -> dict:
    """The reference's own kernels on the host cores (oracle/_ref)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    from particlebase_b200 import workloads as W
    try:
        po.build(ref=True)
    except Exception:
        pass
    s = W.config_c2(seed=2)  # the system rank 0 of the GPU arm times
    steps = max(1, args.steps)
    if po.ref_available():
        R = po.RefKernels(s.box, s.rc, s.r, s.v, s.mass, s.types, [1.0, 1.0], gaussian=True)
        for _ in range(max(1, args.warmup)):
            R.run(DT, 1)  # the first includes the from-scratch sort
        t = time.perf_counter()
        rc = R.run(DT, steps)
        el = time.perf_counter() - t
        kind, cores = "reference", po.ref().ref_threads()
        sample = (f"{steps} steps of the full 1,048,576-atom Gaussian system: the reference's "
                  f"kernels (kernelfuncs.cu, kerneltemplate.hh) compiled for the CPU, "
                  f"one-thread blocks run in parallel by OpenMP; NR rc={rc}")
    else:
        O = po.Oracle(s.box, s.lj, s.rc, s.r, s.v)
        O.run(max(1, args.warmup), DT, mode="gauss")
        t = time.perf_counter()
        O.run(steps, DT, mode="gauss")
        el = time.perf_counter() - t
        kind, cores = "port", po.lib().orc_threads()
        sample = f"{steps} Gaussian steps of the full system, FP64 oracle port"
    v = s.n * steps / el
    return {"metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": 0,
            "steps": steps, "warmup": args.warmup, "higher_is_better": True,
            "config": {"workload": WORKLOAD, "atoms": s.n, "dt": DT},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": kind,
                             "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


# --------------------------------------------------------------------------- GPU arm

def flush_l2(buf):
    buf.zero_()


def run_ours(args, dist: Dist) -> dict:
    import torch
    torch.cuda.set_device(dist.local)
    from particlebase_b200 import workloads as W
    from particlebase_b200.md import from_system
    from particlebase_b200 import _lib as L

    s = W.config_c2(seed=2 + dist.rank)
    half = args.force_kernel == "half"
    p = from_system(s, gaussian=True, fp64_velocities=False, half_shell=half)
    p.clearForce()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > L2

    # warm-up (W steps, rounded up to whole graph units)
    p.run(DT, max(2, args.warmup + (args.warmup % 2)))
    torch.cuda.synchronize()

    steps = args.steps + (args.steps % 2)
    dist.barrier()
    with ClockSampler(torch.cuda.current_device()) as clk:
        t_ms = 0.0
        for _ in range(steps // 2):
            flush_l2(flush)
            torch.cuda.synchronize()
            t_ms += p.run_timed(DT, 2)
        torch.cuda.synchronize()
        warm_ms = p.run_timed(DT, steps)
    dist.barrier()
    clocks = clk.summary()
    status = p.status()
    t_max = dist.reduce(t_ms, "max") / 1e3
    value = replica_rate(dist.ws, s.n, steps, t_max)
    warm_value = s.n * steps / (warm_ms / 1e3)

    # phase breakdown and the force kernel's roofline
    prof = p.profile(DT, 6)
    p.calcBlockID()
    p.calcForce(energy=True)
    ps = p.pair_stats()
    flops = 8.0 * ps["ncand"] + 14.0 * ps["nin"]
    rc_peak = C_double = None
    import ctypes as C
    pk = C.c_double()
    L.check(L.lib().pb_peak_fp32(C.byref(pk)), "peak_fp32")
    fp32_peak = pk.value
    force_s = prof["force"] / 1e3
    achieved = flops / force_s / 1e12
    C_cells = p.grid()[2]
    peaks = measured_peaks()
    hbm = peaks.get("hbm_gbs")
    cells_bytes = 36.0 * s.n + 8.0 * C_cells
    evolve_bytes = 60.0 * s.n
    traffic = profiled_traffic("k_force")

    grid = [int(x) for x in p.grid()[0]]
    build_kernels = p.cell_build_kernels()
    # the device-timed handle is done: the end-to-end leg runs alone, as a
    # driver with one handle would (its memory returns to the pool)
    p.close()

    # e2e through the public API with host buffers (reference driver loop),
    # over the workload's 500 steps (set-up and import included).  The 500
    # host round trips are sensitive to load on the host, so the leg runs
    # three times from scratch and the median time is the value.
    e2e_steps = C2_STEPS
    e2e_times = []
    for _ in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        q = from_system(s, gaussian=True, fp64_velocities=False, half_shell=half)
        q.clearForce()
        temps = []
        for _ in range(e2e_steps):
            q.run(DT, 1)
            temps.append(q.calcTemp())
        r_final = q.getPosition()
        torch.cuda.synchronize()
        e2e_times.append(time.perf_counter() - t0)
        q.close()
    e2e_s = sorted(e2e_times)[1]
    e2e_value = replica_rate(dist.ws, s.n, e2e_steps, dist.reduce(e2e_s, "max"))
    h2d = s.n * (16 + 16 + 4 + 4 + 2)
    d2h = 8 * e2e_steps + r_final.nbytes

    nlist = neighbor_list_leg(s, dist) if dist.rank == 0 else None

    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": dist.ws, "steps": steps,
        "warmup": args.warmup, "ms_per_step": t_max * 1e3 / steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (FP64 reductions)",
        "data": "synthetic fcc lattice + Maxwell-Boltzmann velocities (seeded)",
        "config": {"workload": WORKLOAD, "atoms_per_gpu": s.n, "cells": C_cells,
                   "grid": grid, "dt": DT, "thermostat": "gaussian",
                   "parallelism": f"replicas x{dist.ws}" if dist.ws > 1 else "single",
                   "l2": "flushed (256 MB write) before every timed 2-step graph unit"},
        "warm_l2_value": warm_value,
        "phase_ms": prof,
        "roofline": {"kernel": "k_force_half + k_force_finish" if half else "k_force",
                     "bound": "fp32", "achieved": achieved,
                     "peak": fp32_peak, "unit": "TFLOP/s", "frac": achieved / fp32_peak,
                     "peak_source": "measured FFMA loop (pb_peak_fp32), FP32 non-tensor",
                     "flops_per_atom_step": flops / s.n,
                     "ncand_per_atom": ps["ncand"] / s.n, "nin_per_atom": ps["nin"] / s.n,
                     "traffic": traffic},
        "hbm_kernels": {
            "cell_build": {"alg_bytes": cells_bytes, "ms": prof["cells"],
                           "achieved_gbs": cells_bytes / (prof["cells"] / 1e3) / 1e9,
                           "peak_gbs": hbm, "frac": (cells_bytes / (prof["cells"] / 1e3) / 1e9 / hbm)
                           if hbm else None},
            "evolve": {"alg_bytes": evolve_bytes, "ms": prof["evolve"],
                       "achieved_gbs": evolve_bytes / (prof["evolve"] / 1e3) / 1e9,
                       "peak_gbs": hbm, "frac": (evolve_bytes / (prof["evolve"] / 1e3) / 1e9 / hbm)
                       if hbm else None}},
        "clocks": clocks,
        "device_status": status,
        # per step: the cell build's kernels (2 or 6), the force kernel (+ the
        # fixed-point finish with the half shell), the two Gaussian passes
        "gpu_launches": (build_kernels + (2 if half else 1) + 2) * steps,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d / e2e_steps,
                "d2h_bytes_per_step": d2h / e2e_steps, "steps": e2e_steps,
                "includes": "import from host, per-step pb_md_run + temperature read-back, "
                            "final positions to host",
                "passes_s": [round(t, 4) for t in e2e_times], "reported": "median of 3 passes"},
    }
    if nlist is not None:
        out["neighbor_list"] = nlist
    return out


NL_SKIN = 0.4    # sigma: list radius rc + 0.4
NL_EVERY = 5     # steps between list builds (no atom moves half the skin)


def neighbor_list_leg(s, dist) -> dict:
    """The same system on the Verlet neighbour-list path (cudaParticleMD::useNList
    / makeNList): list radius rc + NL_SKIN, cell list and neighbour list rebuilt
    every NL_EVERY steps; wall-clock time of the rebuilds and the steps."""
    import torch
    from particlebase_b200.md import from_system
    steps = 20 * NL_EVERY
    q = from_system(s, gaussian=True, fp64_velocities=False, cell_rmax=float(s.rc) + NL_SKIN)
    q.useNList(NL_SKIN)
    q.clearForce()
    for _ in range(2):  # warm-up: graphs captured, list buffers sized
        q.makeNList()
        q.run(DT, NL_EVERY)
    torch.cuda.synchronize()
    q.status()
    t0 = time.perf_counter()
    for _ in range(steps // NL_EVERY):
        q.makeNList()
        q.run(DT, NL_EVERY)
    torch.cuda.synchronize()
    t = time.perf_counter() - t0
    info = q.nlist_info()
    status = q.status()
    prof = q.profile(DT, 6)  # no cell build between list builds
    t_build = time.perf_counter()
    for _ in range(5):
        q.makeNList()
    torch.cuda.synchronize()
    build_ms = (time.perf_counter() - t_build) / 5 * 1e3
    q.close()
    return {"metric": "LJ atom-steps/s at 1M atoms, neighbour-list path", "unit": UNIT,
            "value": s.n * steps / t, "ms_per_step": t * 1e3 / steps, "steps": steps,
            "skin": NL_SKIN, "rebuild_every": NL_EVERY, "list_build_ms": build_ms,
            "phase_ms": {"force": prof["force"], "evolve": prof["evolve"]},
            "entries_per_atom": info["mean"], "max_entries": info["max"],
            "device_status": status,
            "timing": "wall clock around the rebuilds and the graph-replayed steps"}


def run_batched(args, dist: Dist) -> dict:
    """256 uneven replicas (N log-uniform in [500, 50,000] as 4k^3 fcc counts,
    density U[0.70, 0.90], T* U[0.7, 1.5], rc 2.5, Gaussian thermostat, FP32
    state with FP64 reductions): all replicas in one batch, whole steps
    replayed from one CUDA graph, force launch shape from the autotuner --
    against the plain path, the same replicas one pb_md handle at a time."""
    import torch
    from particlebase_b200 import workloads as W
    from particlebase_b200.batch import Batch
    from particlebase_b200.md import from_system
    from particlebase_b200.tune import autotune

    steps = args.batch_steps + (args.batch_steps % 2)
    systems = W.uneven_replicas(args.replicas, seed=3 + dist.rank)
    natoms = np.array([s.n for s in systems])
    total = int(natoms.sum())
    tune = autotune(systems, gaussian=True, dt=DT, steps=6, fp64_velocities=False)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")

    b = Batch.from_systems(systems, gaussian=True, dt=DT, fp64_velocities=False,
                           tuning=(tune["threads"], tune["seg_scale"]))
    b.run(max(2, args.warmup + (args.warmup % 2)))
    torch.cuda.synchronize()
    flush.zero_()
    torch.cuda.synchronize()
    dist.barrier()
    batched_ms = b.run_timed(steps)
    status = int(np.bitwise_or.reduce(b.status()))
    prof = b.profile(4)
    b.close()
    batched_ms = dist.reduce(batched_ms, "max")

    # plain path: every replica in its own handle, graph-replayed, one after another
    handles = [from_system(s, gaussian=True, fp64_velocities=False) for s in systems]
    for p in handles:
        p.run(DT, 2)
    torch.cuda.synchronize()
    flush.zero_()
    torch.cuda.synchronize()
    dist.barrier()
    t0 = time.perf_counter()
    plain_ms = 0.0
    for p in handles:
        plain_ms += p.run_timed(DT, steps)
    plain_wall = time.perf_counter() - t0
    for p in handles:
        p.close()
    plain_ms = dist.reduce(plain_ms, "max")

    # end to end through the public API: host state in, all steps, final positions out
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    q = Batch.from_systems(systems, gaussian=True, dt=DT, fp64_velocities=False,
                           tuning=(tune["threads"], tune["seg_scale"]))
    q.run(steps)
    outs = [q.get(k, "r") for k in range(q.nsys)]
    e2e_s = time.perf_counter() - t0
    q.close()
    e2e_s = dist.reduce(e2e_s, "max")

    v_batched = replica_rate(dist.ws, total, steps, batched_ms / 1e3)
    v_plain = replica_rate(dist.ws, total, steps, plain_ms / 1e3)
    return {
        "metric": "batched-replica atom-steps/s (256 uneven LJ replicas)",
        "value": v_batched, "unit": UNIT, "ms_per_step": batched_ms / steps,
        "plain_value": v_plain, "plain_ms_per_step": plain_ms / steps,
        "plain_wall_ms_per_step": plain_wall * 1e3 / steps,
        "speedup_vs_plain": v_batched / v_plain,
        "steps": steps, "replicas": len(systems), "atoms": total,
        "atoms_min": int(natoms.min()), "atoms_max": int(natoms.max()),
        "tuning": {k: tune[k] for k in ("threads", "seg_scale", "cached")},
        "phase_ms": prof, "device_status": status,
        "e2e": {"value": replica_rate(dist.ws, total, steps, e2e_s), "unit": UNIT,
                "h2d_bytes_per_step": total * 42 / steps, "d2h_bytes_per_step": total * 16 / steps,
                "includes": "batch creation from host arrays, all steps, final positions to host"},
        "config": {"workload": "lj_uneven_replicas_256_gauss", "dt": DT, "seed": 3 + dist.rank,
                   "plain": "one pb_md handle per replica, 2-step CUDA graphs, sequential",
                   "l2": "flushed before each timed run; batch state ~0.3 GB > L2"},
    }


def run_served(args, dist: Dist, jobs: int) -> dict:
    """Served MD jobs: a Poisson stream (mean 50 jobs/s) of fcc LJ jobs with N
    log-uniform in [1,000, 200,000] (as 4k^3 counts), density U[0.75, 0.90],
    T* U[0.7, 1.2], steps U[100, 5,000], Gaussian thermostat, submitted in
    real time to the job server under a 120 GB HBM budget.  Latency = done -
    submitted on the server clock (queueing included); throughput = completed
    atom-steps / (last completion - first submission)."""
    import torch
    from particlebase_b200 import workloads as W
    from particlebase_b200.serve import Server

    specs = W.served_jobs(count=jobs, seed=4 + dist.rank)
    free, _ = torch.cuda.mem_get_info()
    budget = min(120e9, 0.8 * free)
    srv = Server(hbm_budget=budget, gaussian=True, fp64_velocities=False, chunk_ms=args.chunk_ms)
    dist.barrier()
    t0 = time.perf_counter()
    ids = []
    lag = 0.0
    for sp in specs:
        delay = sp.arrival - (time.perf_counter() - t0)
        if delay > 0:
            time.sleep(delay)
        else:
            lag = max(lag, -delay)
        ids.append(srv.submit(sp.system(), sp.steps, DT))
    srv.drain()
    infos = [srv.info(i) for i in ids]
    st = srv.stats()
    srv.close()
    lat = np.array([i["t_done"] - i["t_submit"] for i in infos])
    wait = np.array([i["t_admit"] - i["t_submit"] for i in infos])
    span = max(i["t_done"] for i in infos) - min(i["t_submit"] for i in infos)
    atom_steps = float(sum(sp.n * sp.steps for sp in specs))
    status = 0
    for i in infos:
        status |= i["device_status"]
    value = dist.reduce(atom_steps, "sum") / dist.reduce(span, "max")
    return {
        "metric": "served MD jobs: aggregate atom-steps/s and p50/p99 job latency",
        "value": value, "unit": UNIT,
        "p50_latency_s": float(np.percentile(lat, 50)), "p99_latency_s": float(np.percentile(lat, 99)),
        "p50_admission_wait_s": float(np.percentile(wait, 50)),
        "p99_admission_wait_s": float(np.percentile(wait, 99)),
        "jobs": len(specs), "done": st["done"], "failed": st["failed"],
        "atom_steps": atom_steps, "span_s": span,
        "gpu_busy_fraction": st["gpu_seconds"] / span if span > 0 else None,
        "gpu_atom_steps_per_s": atom_steps / st["gpu_seconds"] if st["gpu_seconds"] else None,
        "repacks": st["repacks"], "repack_s": st["repack_seconds"], "chunks": st["chunks"],
        "peak_jobs": st["peak_jobs"], "peak_atoms": st["peak_atoms"],
        "peak_bytes": st["peak_bytes"], "hbm_budget_bytes": budget,
        "submit_lag_s": lag, "device_status": status,
        "config": {"workload": f"lj_served_poisson50_{len(specs)}jobs_gauss", "dt": DT,
                   "seed": 4 + dist.rank, "chunk_ms": args.chunk_ms,
                   "note": "all 2,000 jobs with --workload c4 --jobs 2000"},
    }


def run_kob_andersen(args, dist: Dist) -> dict:
    """Kob-Andersen 80:20 binary mixture, 8,388,608 atoms at density 1.2 from
    uniform random positions, relaxed by 200 capped steepest-descent iterations
    on the GPU (untimed preparation), then a Gaussian thermostat at T* 0.8 with
    FP32 state and FP64 reductions; K timed steps, per-pair cutoffs 2.5 sigma_ab."""
    import torch
    from particlebase_b200 import workloads as W
    from particlebase_b200.md import from_system

    s = W.config_c5(seed=5 + dist.rank, n=args.ka_atoms)
    p = from_system(s, gaussian=True, fp64_velocities=False)
    t0 = time.perf_counter()
    p.minimize(200, 1e-3, 0.02)
    relax_s = time.perf_counter() - t0
    p.clearForce()
    p.adjustVelocities(0.8)
    p.run(DT, max(2, args.warmup + (args.warmup % 2)))
    torch.cuda.synchronize()
    steps = args.ka_steps + (args.ka_steps % 2)
    dist.barrier()
    ms = p.run_timed(DT, steps)
    ms = dist.reduce(ms, "max")
    T = p.calcTemp()
    status = p.status()
    prof = p.profile(DT, 4)
    p.calcBlockID()
    p.calcForce(energy=True)
    ps = p.pair_stats()
    sums = p.sums()
    p.close()
    return {
        "metric": "LJ atom-steps/s, Kob-Andersen 8.4M atoms", "unit": UNIT,
        "value": replica_rate(dist.ws, s.n, steps, ms / 1e3), "ms_per_step": ms / steps, "steps": steps,
        "atoms": s.n, "relax_s": relax_s, "temperature": T, "pe_per_atom": sums["pe"] / s.n,
        "phase_ms": prof, "ncand_per_atom": ps["ncand"] / s.n, "nin_per_atom": ps["nin"] / s.n,
        "flops_per_atom_step": (8 * ps["ncand"] + 14 * ps["nin"]) / s.n,
        "device_status": status,
        "config": {"workload": f"kob_andersen_{s.n}_rho1.2_T0.8_gauss", "dt": DT,
                   "relax": "200 capped steepest-descent iterations (alpha 1e-3, max 0.02 sigma)"},
    }


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-steps", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="all", choices=["all", "c2", "c3", "c4", "c5"],
                    help="c2: 1M-atom single system; c3: batched replicas; c4: served jobs; "
                         "all: the c2 line with c3 under 'batched', c4 under 'served' and "
                         "c5 under 'kob_andersen'")
    ap.add_argument("--jobs", type=int, default=2000,
                    help="served jobs of the C4 stream (default: all 2,000)")
    ap.add_argument("--chunk-ms", type=float, default=100.0)
    ap.add_argument("--ka-atoms", type=int, default=8_388_608)
    ap.add_argument("--ka-steps", type=int, default=300)
    ap.add_argument("--replicas", type=int, default=256)
    ap.add_argument("--batch-steps", type=int, default=200)
    ap.add_argument("--force-kernel", default="full", choices=["full", "half"],
                    help="full: every ordered pair (default); half: every unordered pair once "
                         "(PB_MD_HALF_SHELL)")
    args = ap.parse_args(argv)
    args.warmup = max(3, args.warmup)

    ws, rank, _ = dist_env()
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference_arm(args)), flush=True)
        return 0

    dist = Dist(use_cuda=True)
    try:
        if args.workload in ("c3", "c4", "c5"):
            out = {"c3": lambda: run_batched(args, dist),
                   "c4": lambda: run_served(args, dist, args.jobs),
                   "c5": lambda: run_kob_andersen(args, dist)}[args.workload]()
            if dist.rank == 0:
                print(json.dumps(out), flush=True)
            return 0
        out = run_ours(args, dist)
        if args.workload == "all":
            out["batched"] = run_batched(args, dist)
            out["served"] = run_served(args, dist, args.jobs)
            out["kob_andersen"] = run_kob_andersen(args, dist)
        if dist.rank == 0:
            if dist.ws == 1 and not args.no_cpu_baseline:
                out["cpu_baseline"] = run_cpu_oracle(args.cpu_steps)
            print(json.dumps(out), flush=True)
    finally:
        dist.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
