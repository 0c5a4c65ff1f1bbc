"""The MD job server (pb_srv): continuous batching with exact per-job results.

Bar: every job's final positions, velocities and forces are bit-identical to
the same job run alone through a single-system handle, whatever else was in
the batch while it ran; admission respects the memory budget.
"""
import time

import numpy as np
import pytest

from particlebase_b200 import workloads as W

pytestmark = pytest.mark.gpu

DT = 0.005


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint64 if a.dtype == np.float64 else np.uint32)


def alone(spec, gaussian, fp64_velocities):
    from particlebase_b200.md import from_system
    p = from_system(spec.system(), gaussian=gaussian, fp64_velocities=fp64_velocities)
    p.run(DT, spec.steps)
    v = p.get("vd") if fp64_velocities else p.get("v")
    return p.get("r"), v, p.get("F")


@pytest.mark.parametrize("gaussian,fp64v", [(True, True), (False, False)])
def test_results_same_alone_and_in_the_mix(cuda_lib, gaussian, fp64v):
    from particlebase_b200.serve import Server
    specs = W.served_jobs(count=12, rate=200.0, n_lo=500, n_hi=20_000, steps=(3, 40), seed=21)
    srv = Server(gaussian=gaussian, fp64_velocities=fp64v, chunk_ms=2.0)
    ids = []
    t0 = time.perf_counter()
    for sp in specs:  # arrivals spread over the run, so jobs join a busy batch
        delay = sp.arrival - (time.perf_counter() - t0)
        if delay > 0:
            time.sleep(delay)
        ids.append(srv.submit(sp.system(), sp.steps, DT))
    srv.drain(timeout=300)
    st = srv.stats()
    assert st["done"] == len(specs) and st["failed"] == 0
    assert st["repacks"] >= 2  # the mix changed while jobs were running
    for sp, jid in zip(specs, ids):
        info = srv.info(jid)
        assert info["state"] == "done" and info["device_status"] == 0
        assert info["t_submit"] <= info["t_admit"] <= info["t_done"]
        r, v, F = srv.result(jid)
        ra, va, Fa = alone(sp, gaussian, fp64v)
        assert (bits(r) == bits(ra)).all(), f"job {jid} positions"
        assert (bits(v) == bits(va)).all(), f"job {jid} velocities"
        assert (bits(F) == bits(Fa)).all(), f"job {jid} forces"
    srv.close()


def test_budget_limits_the_resident_set(cuda_lib):
    from particlebase_b200.batch import Batch
    from particlebase_b200.serve import Server
    specs = W.served_jobs(count=6, rate=1e6, n_lo=4000, n_hi=4000, steps=(20, 20), seed=22)
    one = Batch.estimate_bytes([specs[0].system()]) + 4 * specs[0].n
    srv = Server(hbm_budget=int(4.5 * one), gaussian=True, chunk_ms=1.0)
    for sp in specs:
        srv.submit(sp.system(), sp.steps, DT)
    srv.drain(timeout=300)
    st = srv.stats()
    assert st["done"] == 6
    # resident estimates (counting continuing jobs twice while a repack holds
    # both batches) never exceed the budget: at most four of these jobs at once
    assert 2 <= st["peak_jobs"] <= 4
    assert st["peak_bytes"] <= 4.5 * one
    from particlebase_b200 import _lib as L
    big = W.served_jobs(count=1, n_lo=100_000, n_hi=100_000, seed=23)[0]
    with pytest.raises(L.PBError) as e:
        srv.submit(big.system(), 10, DT)
    assert e.value.code == 6  # PB_ERR_OOM
    srv.close()


def test_pool_reserve_and_trim(cuda_lib):
    """pb_pool_reserve takes device memory into the library's pool at once (a
    server does it at creation so that repacks never wait for the pool to
    grow); pb_pool_trim hands the unused part back."""
    import torch
    from particlebase_b200 import _lib as L
    from particlebase_b200.md import from_system
    lib = L.lib()
    assert lib.pb_pool_trim() == 0
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    gb = 1 << 30
    assert lib.pb_pool_reserve(2 * gb) == 0
    free1 = torch.cuda.mem_get_info()[0]
    assert free0 - free1 >= 2 * gb - (64 << 20)
    p = from_system(W.config_c1(), gaussian=True)  # a handle allocates from the reservation
    p.run(DT, 2)
    assert p.status() == 0
    p.close()
    assert lib.pb_pool_trim() == 0
    assert torch.cuda.mem_get_info()[0] >= free0 - (64 << 20)
    # more than the device holds: refused, and nothing is kept
    total = torch.cuda.mem_get_info()[1]
    assert lib.pb_pool_reserve(total + gb) == 6  # PB_ERR_OOM
    assert torch.cuda.mem_get_info()[0] >= free0 - (64 << 20)
