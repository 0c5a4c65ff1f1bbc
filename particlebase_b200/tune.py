"""Autotuner for the force launch of a batch: threads per CTA and z-run length.

The force kernel's work item is one column run of `seg` z cells of one
system (its cell tile: 3 x 3 columns x (seg + 2) cells staged in shared
memory); `seg` is chosen per system from its mean cell occupancy to give
about 160 home atoms per CTA, times a scale.  The tuner times whole steps of
the batch for each (threads, scale) candidate and keeps the fastest.  Both
parameters change only how the work is split into CTAs, not which pairs are
computed.  Results are cached in a JSON file keyed by the device name, the
integration mode and a coarse signature of the batch (system count and atom
count histogram), so a recurring batch shape is tuned once.

The cache file is $PB_TUNE_CACHE, else ~/.cache/particlebase_b200/tune.json.
"""
from __future__ import annotations

import json
import math
import os
from typing import Sequence

import numpy as np

from .batch import Batch
from .workloads import LJSystem

CANDIDATES = [(256, 1.0), (128, 1.0), (256, 0.5), (256, 0.75), (256, 1.5), (256, 2.0),
              (128, 0.5), (128, 1.5)]


def cache_path() -> str:
    return os.environ.get("PB_TUNE_CACHE") or os.path.join(
        os.path.expanduser("~"), ".cache", "particlebase_b200", "tune.json")


def _device_name() -> str:
    try:
        import torch
        return torch.cuda.get_device_name()
    except Exception:
        return "cuda"


def signature(systems: Sequence[LJSystem], gaussian: bool) -> str:
    """Device, mode, system count (log2 bucket) and atoms-per-system histogram
    over log2 buckets -- batches with the same signature share a tuning."""
    n = np.array([s.n for s in systems], np.float64)
    hist = np.bincount(np.floor(np.log2(n)).astype(int), minlength=24)[:24]
    frac = np.round(hist / max(1, len(n)), 1)
    return json.dumps({"dev": _device_name(), "gauss": bool(gaussian),
                       "nsys": int(math.log2(max(1, len(n)))),
                       "hist": [float(x) for x in frac]}, sort_keys=True)


def _load(path: str) -> dict:
    try:
        with open(path) as fh:
            return json.load(fh)
    except Exception:
        return {}


def _store(path: str, table: dict) -> None:
    os.makedirs(os.path.dirname(path), exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as fh:
        json.dump(table, fh, indent=1, sort_keys=True)
    os.replace(tmp, path)


def autotune(systems: Sequence[LJSystem], gaussian: bool = False, dt: float = 0.005,
             steps: int = 6, candidates=CANDIDATES, use_cache: bool = True,
             fp64_velocities: bool | None = None) -> dict:
    """Best (threads, seg_scale) for this batch shape; returns
    {"threads", "seg_scale", "ms_per_step", "trials": [...], "cached": bool}."""
    path = cache_path()
    key = signature(systems, gaussian)
    table = _load(path) if use_cache else {}
    if use_cache and key in table:
        hit = dict(table[key])
        hit["cached"] = True
        return hit
    b = Batch.from_systems(systems, gaussian=gaussian, dt=dt, fp64_velocities=fp64_velocities)
    trials = []
    try:
        for threads, scale in candidates:
            b.set_tuning(threads, scale)
            b.setup_cells()
            b.run(2)  # graph capture + warm
            ms = b.run_timed(steps) / steps
            trials.append({"threads": threads, "seg_scale": scale, "ms_per_step": ms})
    finally:
        b.close()
    best = min(trials, key=lambda t: t["ms_per_step"])
    res = {"threads": best["threads"], "seg_scale": best["seg_scale"],
           "ms_per_step": best["ms_per_step"], "trials": trials}
    if use_cache:
        table = _load(path)
        table[key] = res
        try:
            _store(path, table)
        except OSError:
            pass
    res = dict(res)
    res["cached"] = False
    return res
