"""The half-shell force kernel (PB_MD_HALF_SHELL): every unordered pair once,
Newton's third law, force sums in exact 64-bit fixed point.

Bars: forces within 1e-5 relative RMS of the FP64 oracle (C1, 1M atoms, the
Kob-Andersen mixture with per-pair cutoffs, a 3-cell box); potential energy,
virial and pair count equal to the full-shell kernel's within FP32 rounding;
every system of a batch bit-identical to its run alone; extreme but finite
forces (a random clump) exact through the coarse sums; status bits as the
full-shell kernel raises them.
"""
import numpy as np
import pytest

from particlebase_b200 import workloads as W

pytestmark = pytest.mark.gpu

FORCE_RELRMS = 1e-5
DT = 0.005


def relrms(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


def perturbed(s, amp, seed):
    rng = np.random.default_rng(seed)
    r = np.mod(s.r + rng.uniform(-amp, amp, s.r.shape), s.L)
    s.r = np.minimum(r.astype(np.float32), np.nextafter(np.float32(s.L), np.float32(0)))
    s.r = s.r.astype(np.float64)
    return s


def half(s, **kw):
    from particlebase_b200.md import from_system
    return from_system(s, half_shell=True, **kw)


def oracle_F(po, s, r4):
    O = po.Oracle(s.box, s.lj, s.rc, r4[:, :3].astype(np.float64), types=s.types)
    info = O.forces()
    return O.get("F"), info


@pytest.mark.parametrize("make", [
    lambda: perturbed(W.config_c1(), 0.1, 5),
    lambda: perturbed(W.config_c2(), 0.1, 6),
    lambda: W.kob_andersen_random(6000, 1.2, 0.8, seed=9),
    lambda: perturbed(W.fcc_system(5, 0.8442, 0.72, seed=1), 0.1, 7),  # 3 x 3 x 3 cells
], ids=["c1", "1m", "kob_andersen", "three_cells"])
def test_forces_vs_oracle(cuda_lib, po, make):
    s = make()
    p = half(s)
    if s.ntypes > 1:
        p.minimize(50, 1e-3, 0.02)  # relax the random start, as C5 does
    p.calcBlockID()
    p.calcForce(energy=True)
    F = p.get("F")[:, :3].astype(np.float64)
    Fo, info = oracle_F(po, s, p.get("r"))
    assert relrms(F, Fo) < FORCE_RELRMS
    sums = p.sums()
    assert sums["pe"] == pytest.approx(info["pe"], rel=1e-6, abs=1e-6 * s.n)
    # pairs at the cutoff to within FP32 rounding of the distance
    assert p.pair_stats()["nin"] == pytest.approx(info["nin"], rel=1e-6, abs=2)
    assert p.status() == 0


def test_same_energy_as_full_shell(cuda_lib):
    from particlebase_b200.md import from_system
    s = perturbed(W.config_c1(), 0.1, 8)
    a, b = half(s), from_system(s)
    for p in (a, b):
        p.calcBlockID()
        p.calcForce(energy=True)
    sa, sb = a.sums(), b.sums()
    for k in ("pe", "pe_shift", "virial"):
        assert sa[k] == pytest.approx(sb[k], rel=1e-6)
    assert a.pair_stats()["nin"] == b.pair_stats()["nin"]
    assert relrms(a.get("F")[:, :3].astype(np.float64), b.get("F")[:, :3].astype(np.float64)) < 1e-6


def test_runs_are_bit_identical(cuda_lib):
    s = perturbed(W.config_c1(), 0.05, 9)
    out = []
    for _ in range(2):
        p = half(s)
        p.clearForce()
        p.run(DT, 20)
        out.append((p.get("r"), p.get("v"), p.get("F")))
    for x, y in zip(*out):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("gaussian", [False, True])
def test_batch_equals_alone(cuda_lib, gaussian):
    from particlebase_b200.batch import Batch
    systems = W.uneven_replicas(count=6, n_lo=500, n_hi=6000, seed=11)
    b = Batch.from_systems(systems, gaussian=gaussian, dt=DT, half_shell=True)
    b.run(10)
    assert (b.status() == 0).all()
    vf = "vd" if gaussian else "v"
    for k, s in enumerate(systems):
        p = half(s, gaussian=gaussian)
        p.run(DT, 10)
        for f in ("r", vf, "F", "Fold"):
            assert np.array_equal(b.get(k, f), p.get(f)), f"system {k} {f}"


def test_extreme_forces_stay_exact(cuda_lib, po):
    """A clump of 60 atoms in a 2.4-sigma cube: pair forces up to ~1e9 go to
    the coarse fixed-point sums and still match the oracle."""
    rng = np.random.default_rng(2)
    L = 30.0
    gas = rng.uniform(0, L, (800, 3))
    clump = 15.0 + rng.uniform(0, 2.4, (60, 3))
    r = np.concatenate([gas, clump])
    box = np.array([0, L, 0, L, 0, L], np.float32)
    s = W.LJSystem(box=box, r=r, v=np.zeros_like(r), mass=np.ones(len(r)),
                   types=np.zeros(len(r), np.uint32), lj=W.single_type_lj(), rc=2.5)
    p = half(s)
    p.calcBlockID()
    p.calcForce()
    Fo, _ = oracle_F(po, s, p.get("r"))
    assert relrms(p.get("F")[:, :3].astype(np.float64), Fo) < FORCE_RELRMS


def test_wait_timeout_is_reported_and_the_handle_recovers(cuda_lib, po):
    s = perturbed(W.config_c1(), 0.05, 3)
    p = half(s)
    p.calcBlockID()
    p.force_wait_test(2000)
    assert p.status() & 0x4
    p.calcForce()
    assert p.status() == 0
    Fo, _ = oracle_F(po, s, p.get("r"))
    assert relrms(p.get("F")[:, :3].astype(np.float64), Fo) < FORCE_RELRMS
