"""Accuracy of every benchmark configuration against the FP64 oracle.

For each configuration: force relative RMS error of the FP32 path (and of the
FP64-accumulation option) against the oracle on the same FP32 positions, and
the NVE energy drift (epsilon per atom per 1000 velocity-Verlet steps, fit
over steps 1..1000, shifted-potential energy plus kinetic energy).  Bars:
force error <= 1e-5; drift within 5e-5 of the FP64 oracle's drift from the
same start where the oracle runs it (C1, every C3 replica and C4 job tested),
else drift <= 1e-4.  A system of a few hundred atoms drifts by about 1e-4 in
the oracle itself (truncated force), so the bar there is the difference the
FP32 path adds.  With PB_ACCURACY_OUT set, the measured figures are written
there as JSON.
"""
import json
import os

import numpy as np
import pytest

from particlebase_b200 import workloads as W

pytestmark = pytest.mark.gpu

FORCE_RELRMS = 1e-5
DRIFT = 1e-4
DRIFT_VS_ORACLE = 5e-5
DT = 0.005
RESULTS = {}


def relrms(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


def perturbed(s, amp=0.1, seed=0):
    rng = np.random.default_rng(seed)
    L = s.L
    r = np.mod(s.r + rng.uniform(-amp, amp, s.r.shape), L).astype(np.float32)
    s.r = np.minimum(r, np.nextafter(L.astype(np.float32), np.float32(0))).astype(np.float64)
    return s


def force_errors(po, s):
    from particlebase_b200.md import from_system
    O = po.Oracle(s.box, s.lj, s.rc, s.r.astype(np.float32).astype(np.float64), types=s.types)
    O.forces()
    Fo = O.get("F")
    out = {}
    for acc64 in (False, True):
        p = from_system(s, fp64_forces=acc64)
        p.calcBlockID()
        p.calcForce()
        out["fp64_acc" if acc64 else "fp32_acc"] = relrms(p.get("F")[:, :3].astype(np.float64), Fo)
        p.close()
    return out


def nve_drift(p, steps=1000):
    """Energy per atom after each step; drift = slope of a linear fit x 1000
    (step 0 excluded: it starts from Fold = 0, the reference's clearForce)."""
    e = []
    p.clearForce()
    for _ in range(steps + 1):
        p.calcBlockID()
        p.calcForce(energy=True)
        pe = p.sums()["pe_shift"]
        p.TimeEvolution(DT)
        p.treatPeriodicCondition()
        e.append(0.5 * p.sums()["mv2"] + pe)
    e = np.array(e[1:]) / p.n
    return float(np.polyfit(np.arange(len(e)), e, 1)[0] * 1000), float(e.std())


def oracle_drift(po, s, steps=1000):
    """The FP64 oracle's NVE drift on the same start, same definition: energy
    per atom at t_k from the force evaluation at r(t_k) and v(t_k), steps
    1..steps fitted (orc_run records both)."""
    O = po.Oracle(s.box, s.lj, s.rc, s.r, s.v, s.mass, s.types)
    e = O.run(steps + 1, DT, record=True)
    tot = (e[1:, 0] + e[1:, 2]) / s.n
    return float(np.polyfit(np.arange(len(tot)), tot, 1)[0] * 1000)


def record(name, **kw):
    RESULTS[name] = kw
    out = os.environ.get("PB_ACCURACY_OUT")
    if out:
        with open(out, "w") as fh:
            json.dump(RESULTS, fh, indent=1)


def check(name, forces, drift, spread, odrift=None):
    """drift, odrift: one system's figures, or lists over the systems of a batch."""
    record(name, force_relrms=forces, nve_drift_per_1000=drift, energy_std=spread,
           oracle_nve_drift_per_1000=odrift)
    assert forces["fp32_acc"] < FORCE_RELRMS and forces["fp64_acc"] < FORCE_RELRMS, forces
    if odrift is None:
        assert abs(drift) < DRIFT, drift
        return
    d = np.atleast_1d(drift)
    o = np.atleast_1d(odrift)
    assert np.all(np.abs(d - o) < DRIFT_VS_ORACLE), list(zip(d, o))


def test_accuracy_c1(cuda_lib, po):
    from particlebase_b200.md import from_system
    s = W.config_c1()
    forces = force_errors(po, perturbed(W.config_c1(), seed=11))
    drift, spread = nve_drift(from_system(s))
    check("C1 fcc 4,000", forces, drift, spread, oracle_drift(po, W.config_c1()))


def test_accuracy_c2(cuda_lib, po):
    from particlebase_b200.md import from_system
    forces = force_errors(po, perturbed(W.config_c2(), seed=12))
    drift, spread = nve_drift(from_system(W.config_c2()))
    check("C2 fcc 1,048,576", forces, drift, spread)


def _batch_drift(systems, steps=1000):
    """NVE drift of every system of one batch (VV, FP32 velocities)."""
    from particlebase_b200.batch import Batch
    b = Batch.from_systems(systems, dt=DT)
    b.clear_force()
    e = []
    for _ in range(steps + 1):
        b.force(energy=True)
        pe = b.sums()[:, 3]
        b.run(1)
        mv2 = b.sums()[:, 0]
        e.append(0.5 * mv2 + pe)
    e = (np.array(e[1:]) / np.array([s.n for s in systems])[None, :])
    drifts = [float(np.polyfit(np.arange(len(e)), e[:, k], 1)[0] * 1000) for k in range(len(systems))]
    b.close()
    return drifts, float(e.std(0).max())


def test_accuracy_c3_replicas(cuda_lib, po):
    systems = W.uneven_replicas(256, seed=3)[::32]  # 8 of the 256 benchmark replicas
    worst = {"fp32_acc": 0.0, "fp64_acc": 0.0}
    for k, s in enumerate(systems):
        f = force_errors(po, perturbed(W.uneven_replicas(256, seed=3)[32 * k], seed=20 + k))
        worst = {m: max(worst[m], f[m]) for m in worst}
    drifts, spread = _batch_drift(systems)
    # the oracle's drift on each of them, from the same start
    odrifts = [oracle_drift(po, s) for s in W.uneven_replicas(256, seed=3)[::32]]
    check("C3 uneven replicas (8 of 256, batched)", worst, drifts, spread, odrifts)
    record("C3 replica atoms", atoms=[s.n for s in systems])


def test_accuracy_c4_jobs(cuda_lib, po):
    specs = W.served_jobs(count=40, seed=4)[::10]  # 4 jobs of the served stream
    systems = [sp.system() for sp in specs]
    worst = {"fp32_acc": 0.0, "fp64_acc": 0.0}
    for k, sp in enumerate(specs):
        f = force_errors(po, perturbed(sp.system(), seed=30 + k))
        worst = {m: max(worst[m], f[m]) for m in worst}
    drifts, spread = _batch_drift(systems)
    odrifts = [oracle_drift(po, sp.system()) for sp in specs]
    check("C4 served jobs (4 of the stream, batched)", worst, drifts, spread, odrifts)
    record("C4 job atoms", atoms=[s.n for s in systems])


@pytest.mark.slow
def test_accuracy_c5_kob_andersen(cuda_lib, po):
    """8.4M-atom Kob-Andersen mixture: relaxed on the GPU (200 capped
    steepest-descent iterations), thermalised 300 Gaussian steps, then forces
    against the oracle and 1000 NVE steps."""
    from particlebase_b200.md import from_system
    s = W.config_c5()
    p = from_system(s, gaussian=True, fp64_velocities=False)
    p.minimize(200, 1e-3, 0.02)
    p.clearForce()
    p.adjustVelocities(0.8)
    p.run(DT, 300)
    s.r = p.get("r")[:, :3].astype(np.float64)
    s.v = p.velocities()
    p.close()
    forces = force_errors(po, s)
    q = from_system(s)  # NVE from the thermalised state
    drift, spread = nve_drift(q)
    check("C5 Kob-Andersen 8,388,608", forces, drift, spread)
