"""Batches of independent systems (pb_batch) against single-system handles
and the oracle.

Bars: every system of a batch is bit-identical to the same system run alone
(positions, velocities, forces, Gaussian friction), including across a
repack that retires and admits systems mid-run; forces of every system
within 1e-5 relative RMS of the FP64 oracle; status bits raised per system.
"""
import numpy as np
import pytest

from particlebase_b200 import workloads as W

pytestmark = pytest.mark.gpu

FORCE_RELRMS = 1e-5
DT = 0.005


def relrms(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


def replicas(count, seed, n_hi=6000):
    return W.uneven_replicas(count=count, n_lo=500, n_hi=n_hi, seed=seed)


def perturbed(systems, amp=0.1, seed=0):
    """Displace lattice sites so forces are O(1) (a perfect fcc lattice has
    near-zero net forces, where a relative error measures only cancellation)."""
    rng = np.random.default_rng(seed)
    for s in systems:
        L = s.L
        r = np.mod(s.r + rng.uniform(-amp, amp, s.r.shape), L).astype(np.float32)
        r = np.minimum(r, np.nextafter(L.astype(np.float32), np.float32(0)))
        s.r = r.astype(np.float64)
    return systems


def alone_md(s, gaussian):
    from particlebase_b200.md import from_system
    return from_system(s, gaussian=gaussian)


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint64 if a.dtype == np.float64 else np.uint32)


def assert_same(a, b, what):
    assert a.shape == b.shape, what
    same = bits(a) == bits(b)
    assert same.all(), f"{what}: {int((~same).sum())} of {same.size} values differ"


@pytest.mark.parametrize("gaussian", [False, True])
def test_batch_equals_alone(cuda_lib, gaussian):
    from particlebase_b200.batch import Batch
    systems = replicas(6, seed=11)
    b = Batch.from_systems(systems, gaussian=gaussian, dt=DT)
    b.run(10)
    assert (b.status() == 0).all()
    xi = b.sums()[:, 5]
    for k, s in enumerate(systems):
        p = alone_md(s, gaussian)
        p.run(DT, 10)
        assert_same(b.get(k, "r"), p.get("r"), f"system {k} positions")
        vf = "vd" if gaussian else "v"
        assert_same(b.get(k, vf), p.get(vf), f"system {k} velocities")
        assert_same(b.get(k, "F"), p.get("F"), f"system {k} forces")
        assert_same(b.get(k, "Fold"), p.get("Fold"), f"system {k} previous forces")
        if gaussian:
            assert xi[k] == p.sums()["xi"], f"system {k} friction"


def test_batch_forces_vs_oracle(cuda_lib, po):
    from particlebase_b200.batch import Batch
    systems = perturbed(replicas(4, seed=12))
    systems.append(W.kob_andersen_random(3000, 1.2, 0.8, seed=5))  # two types, per-pair rc
    for s in systems:
        s.r = s.r.astype(np.float32).astype(np.float64)
    b = Batch.from_systems(systems, dt=DT)
    b.force(energy=True)
    sums = b.sums()
    for k, s in enumerate(systems):
        O = po.Oracle(s.box, s.lj, s.rc, s.r, types=s.types)
        info = O.forces()
        F = b.get(k, "F")[:, :3].astype(np.float64)
        assert relrms(F, O.get("F")) < FORCE_RELRMS, f"system {k}"
        assert abs(sums[k, 2] - info["pe"]) <= 1e-5 * abs(info["pe"]) + 1e-6, f"pe {k}"


def test_repack_continues_bitwise(cuda_lib):
    """Systems that stay through a repack, and systems admitted by it, follow
    the same trajectory as when run alone from the start."""
    from particlebase_b200.batch import Batch
    systems = replicas(4, seed=13)
    a = Batch.from_systems(systems[:3], gaussian=True, dt=DT)
    a.run(4)
    b = a.repack([2, -1, 0], {1: systems[3]}, dt=DT)
    a.close()
    b.run(6)
    for slot, (s, steps) in {0: (systems[2], 10), 1: (systems[3], 6), 2: (systems[0], 10)}.items():
        p = alone_md(s, True)
        p.run(DT, steps)
        assert_same(b.get(slot, "r"), p.get("r"), f"slot {slot} positions")
        assert_same(b.get(slot, "vd"), p.get("vd"), f"slot {slot} velocities")
        assert b.sums()[slot, 5] == p.sums()["xi"], f"slot {slot} friction"


def test_status_is_per_system(cuda_lib, po):
    """A dense ball in one system overflows its force stage; only that system's
    status word reports it, and its forces stay correct."""
    from particlebase_b200.batch import Batch
    rng = np.random.default_rng(4)
    L = 40.0
    r = np.mod(np.concatenate([rng.uniform(0, L, (2000, 3)), 20.0 + rng.normal(0, 1.5, (3000, 3))]), L)
    r = r.astype(np.float32).astype(np.float64)
    box = np.array([0, L, 0, L, 0, L], np.float32)
    dense = W.LJSystem(box=box, r=r, v=np.zeros_like(r), mass=np.ones(len(r)),
                       types=np.zeros(len(r), np.uint32), lj=W.single_type_lj(), rc=2.5)
    systems = [perturbed(replicas(1, seed=14))[0], dense, perturbed(replicas(1, seed=15))[0]]
    b = Batch.from_systems(systems, dt=DT)
    b.status()
    b.force()
    st = b.status()
    assert st[1] & 1 and st[0] == 0 and st[2] == 0
    O = po.Oracle(box, dense.lj, dense.rc, r, types=dense.types)
    O.forces()
    assert relrms(b.get(1, "F")[:, :3].astype(np.float64), O.get("F")) < FORCE_RELRMS


def test_tuning_keeps_forces(cuda_lib, po):
    """Force launch tuning (threads per CTA, z-run length) changes the work
    split, not the physics: forces stay within the oracle bar."""
    from particlebase_b200.batch import Batch
    systems = perturbed(replicas(3, seed=16))
    for threads, scale in [(128, 0.5), (256, 2.0)]:
        b = Batch.from_systems(systems, dt=DT, tuning=(threads, scale))
        b.force()
        for k, s in enumerate(systems):
            O = po.Oracle(s.box, s.lj, s.rc, s.r, types=s.types)
            O.forces()
            assert relrms(b.get(k, "F")[:, :3].astype(np.float64), O.get("F")) < FORCE_RELRMS


def test_batch_velocity_control(cuda_lib):
    from particlebase_b200.batch import Batch
    systems = replicas(3, seed=17)
    b = Batch.from_systems(systems, dt=DT)
    T0 = b.temperatures()
    assert np.allclose(T0, [s.temperature for s in systems], rtol=1e-5)
    b.scale_velocities([1.0, 2.0, 0.5])
    T1 = b.temperatures()
    assert np.allclose(T1 / T0, [1.0, 4.0, 0.25], rtol=1e-5)
    b.adjust_velocities([1.0, 1.0, 1.0])
    for k in range(3):
        v = b.velocities(k)
        assert np.allclose(v.mean(0), 0, atol=1e-5) and np.allclose(v.std(0), 1.0, rtol=1e-4)


def test_batch_errors(cuda_lib):
    from particlebase_b200 import _lib as L
    from particlebase_b200.batch import Batch
    b = Batch([100, 200])
    with pytest.raises(L.PBError) as e:
        b.setup_cells()
    assert e.value.code == 3
    with pytest.raises(L.PBError) as e:
        b.set_system(0, [0, 5, 0, 5, 0, 5], 2.5, [1.0, 1.0], 9, DT)  # ntypes > 8
    assert e.value.code == 1
    out = np.empty(400, np.float32)
    assert cuda_lib.pb_batch_get(b.h, 5, 0, out.ctypes.data, out.nbytes) == 1  # no system 5


def test_step_budgets_stop_each_system_exactly(cuda_lib):
    """Systems with different step budgets share graph replays; each stops after
    exactly its own count and then matches its alone run of that many steps."""
    from particlebase_b200.batch import Batch
    systems = replicas(4, seed=18)
    budgets = [3, 10, 0, 7]
    for gaussian in (False, True):
        b = Batch.from_systems(systems, gaussian=gaussian, dt=DT)
        b.set_steps_left(budgets)
        b.run(12)
        assert list(b.steps_left()) == [0, 0, 0, 0]
        vf = "vd" if gaussian else "v"
        for k, s in enumerate(systems):
            p = alone_md(s, gaussian)
            if budgets[k]:
                p.run(DT, budgets[k])
            assert_same(b.get(k, "r"), p.get("r"), f"system {k} positions")
            assert_same(b.get(k, vf), p.get(vf), f"system {k} velocities")
            assert_same(b.get(k, "F"), p.get("F"), f"system {k} last force")
        b.close()


@pytest.mark.parametrize("gaussian", [False, True])
def test_nonfinite_replica_is_isolated(cuda_lib, gaussian):
    """Failure detection made on the host: one atom of the middle replica gets a
    NaN velocity before import (the reference drivers stop on a NaN temperature,
    testMD2.cu:157-163).  Only that replica raises PB_STATUS_NONFINITE; the
    others stay bit-identical to their runs alone, and the NaN atom's position,
    binned to cell 0 of its own box, breaks no cell list."""
    import copy

    from particlebase_b200.batch import Batch
    systems = replicas(3, seed=31, n_hi=3000)
    bad = copy.deepcopy(systems[1])
    bad.v = bad.v.copy()
    bad.v[0, 0] = np.nan
    b = Batch.from_systems([systems[0], bad, systems[2]], gaussian=gaussian, dt=DT)
    b.run(6)
    st = b.status()
    assert st[1] & 0x2, "the NaN replica raises PB_STATUS_NONFINITE"
    assert st[0] == 0 and st[2] == 0
    vf = "vd" if gaussian else "v"
    for k in (0, 2):
        p = alone_md(systems[k], gaussian)
        p.run(DT, 6)
        assert_same(b.get(k, "r"), p.get("r"), f"system {k} positions")
        assert_same(b.get(k, vf), p.get(vf), f"system {k} velocities")
    r1 = b.get(1, "r")[:, :3]
    assert np.isnan(r1[0]).any()
    if not gaussian:
        # velocity Verlet: the NaN atom takes part in no pair (its distances
        # compare false), so the replica's other atoms stay finite; the
        # Gaussian friction couples every atom and spreads the NaN instead
        assert np.isfinite(r1[1:]).all()
