"""Verlet neighbour-list path (cudaParticleMD::useNList / makeNList and the list
branch of calcForce, cudaParticleMD.cu:41-44, 338-394) against the oracle and
against the cell-list path.

Bars: forces within 1e-5 relative RMS of the FP64 oracle; potential energy
within 1e-5 relative of the oracle; a short trajectory with periodic list
rebuilds within 1e-4 sigma of the cell-list trajectory; a list that outlives
its skin is reported, not silently used.
"""
import numpy as np
import pytest

from particlebase_b200 import workloads as W

pytestmark = pytest.mark.gpu

FORCE_RELRMS = 1e-5
SKIN = 0.3
DT = 0.005
STALE = 0x40  # PB_STATUS_STALE_NLIST


def relrms(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


def perturbed(s, amp, seed):
    rng = np.random.default_rng(seed)
    r = np.mod(s.r + rng.uniform(-amp, amp, s.r.shape), s.L)
    s.r = r.astype(np.float32).astype(np.float64)
    return s


def with_list(s, skin=SKIN, gaussian=False):
    from particlebase_b200.md import from_system
    p = from_system(s, gaussian=gaussian, cell_rmax=float(s.rc) + skin)
    p.useNList(skin)
    p.makeNList()
    return p


@pytest.mark.parametrize("system", ["fcc", "kob_andersen"])
def test_list_forces_vs_oracle(cuda_lib, po, system):
    if system == "fcc":
        s = perturbed(W.fcc_system(8, 0.8442, 0.72, seed=21), 0.1, 22)
    else:
        s = W.kob_andersen_random(3000, 1.2, 0.8, seed=23)
        s.r = s.r.astype(np.float32).astype(np.float64)
    p = with_list(s)
    info = p.nlist_info()
    assert 0 < info["mean"] <= info["max"] <= info["capacity"]
    p.calcForce(energy=True)
    F = p.get("F")[:, :3].astype(np.float64)
    O = po.Oracle(s.box, s.lj, s.rc, s.r, types=s.types)
    oinfo = O.forces()
    assert relrms(F, O.get("F")) < FORCE_RELRMS
    pe = p.sums()["pe"]
    assert abs(pe - oinfo["pe"]) <= 1e-5 * abs(oinfo["pe"]) + 1e-6
    assert p.status() == 0


def test_list_trajectory_matches_cell_path(cuda_lib):
    from particlebase_b200.md import from_system
    s = perturbed(W.fcc_system(8, 0.8442, 0.72, seed=31), 0.05, 32)
    # rebuilt every 5 steps with a 0.4 sigma skin: at T* = 0.72 no atom moves
    # half the skin between builds, so the list stays valid (status clean)
    a = with_list(s, skin=0.4, gaussian=True)
    a.clearForce()
    for _ in range(8):
        a.makeNList()
        a.run(DT, 5)
    assert a.status() == 0
    b = from_system(s, gaussian=True)
    b.clearForce()
    b.run(DT, 40)
    d = a.get("r")[:, :3].astype(np.float64) - b.get("r")[:, :3].astype(np.float64)
    d -= s.L * np.round(d / s.L)
    assert np.abs(d).max() < 1e-4
    assert abs(a.sums()["xi"] - b.sums()["xi"]) < 1e-4


def test_stale_list_is_reported(cuda_lib):
    s = perturbed(W.fcc_system(8, 0.8442, 0.72, seed=41), 0.05, 42)
    p = with_list(s, skin=0.02)
    p.clearForce()
    p.run(DT, 40)  # atoms move ~0.2 sigma: far more than half the skin
    assert p.status() & STALE
    p.makeNList()
    p.calcForce()
    assert p.status() == 0


def test_list_needs_cells_as_wide_as_its_radius(cuda_lib):
    from particlebase_b200.md import from_system
    s = W.fcc_system(8, 0.8442, 0.72, seed=51)
    p = from_system(s)  # cells sized for the cutoff only
    p.useNList(SKIN)
    with pytest.raises(Exception):
        p.makeNList()
    p.useNList(-1.0)  # back to the cell list
    p.calcForce()
