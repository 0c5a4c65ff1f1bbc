"""Parity of the CUDA path (through the C ABI) with the oracle.

Bars: cell assignment, per-cell member sets and the 27-neighbour table are
bit-exact; forces within 1e-5 relative RMS of the FP64 oracle (FP32 path);
trajectories and energies within the tolerances stated per test.
"""
import numpy as np
import pytest

from particlebase_b200 import workloads as W

pytestmark = pytest.mark.gpu

FORCE_RELRMS = 1e-5


def relrms(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


def md(cuda_lib, s, **kw):
    from particlebase_b200.md import from_system
    return from_system(s, **kw)


def perturbed(s, amp, seed):
    rng = np.random.default_rng(seed)
    r = s.r + rng.uniform(-amp, amp, s.r.shape)
    L = s.L
    r = np.mod(r, L)
    r = np.minimum(r.astype(np.float32), np.nextafter(np.float32(L), np.float32(0)))
    s.r = r.astype(np.float64)
    return s


def oracle_forces(po, s, r4=None):
    r = s.r if r4 is None else r4[:, :3].astype(np.float64)
    O = po.Oracle(s.box, s.lj, s.rc, r.astype(np.float32).astype(np.float64), types=s.types)
    info = O.forces()
    return O.get("F"), info


def check_cells(p, s, po):
    r4 = p.get("r")
    cid = p.get("cell_of")
    assert np.array_equal(cid, po.bin_cells(r4, s.box, s.rc)), "cell of each atom"
    n3, ln, C = p.grid()
    on, oln = po.grid(s.box, s.rc)
    assert np.array_equal(n3, on) and np.array_equal(ln, oln)
    assert np.array_equal(p.get("neighbors"), po.neighbor_table(s.box, s.rc))
    key = p.get("cell_key")
    start = p.get("cell_start")
    pid = p.get("pid")
    assert start[-1] == s.n
    assert np.array_equal(np.sort(pid), np.arange(s.n))
    ostart, omem = po.cell_list(cid, C, r4[:, 2])
    for ref in range(C):
        k = key[ref]
        got = pid[start[k]:start[k + 1]]
        exp = omem[ostart[ref]:ostart[ref + 1]]
        assert np.array_equal(got, exp), f"members of cell {ref}"  # same set, same z order
    rs = p.get("r_sorted")
    assert np.array_equal(rs[:, :3].view(np.uint32), r4[pid, :3].view(np.uint32))
    assert np.array_equal(rs[:, 3].view(np.int32), s.types[pid].astype(np.int32))


def test_cells_bit_exact_c1(cuda_lib, po, golden):
    s = W.config_c1()
    s.r = golden["c1_r4"][:, :3].astype(np.float64)
    p = md(cuda_lib, s)
    p.calcBlockID()
    assert np.array_equal(p.get("cell_of"), golden["c1_cell_of"])
    assert np.array_equal(p.get("neighbors"), golden["c1_neighbors"])
    check_cells(p, s, po)


def test_cells_bit_exact_1m(cuda_lib, po):
    s = perturbed(W.config_c2(), 0.1, 7)
    p = md(cuda_lib, s, gaussian=True)
    p.calcBlockID()
    # the same checks as at C1: cell of every atom, grid, 27-neighbour table,
    # per-cell member sets in canonical (z, id) order, sorted positions
    check_cells(p, s, po)


@pytest.mark.parametrize("shuffle", [False, True])
def test_bucket_and_sort_builds_agree(cuda_lib, po, shuffle, monkeypatch):
    """The engine picks the faster of its two cell builds at set-up; both must
    give the same bits.  A 256,000-atom lattice in lattice order (the bucket
    build's case) and in random particle order (the counting sort's), each
    built both ways; the sorted layout, cell starts, force-kernel mirrors and
    forces are compared, and the first build is checked against the oracle."""
    s = perturbed(W.fcc_system(40, 0.8442, 0.72, seed=9), 0.1, 8)
    if shuffle:
        perm = np.random.default_rng(3).permutation(s.n)
        s.r, s.v = s.r[perm], s.v[perm]
    got = []
    for mode in ("bucket", "sort"):
        monkeypatch.setenv("PB_CELL_BUILD", mode)
        p = md(cuda_lib, s)
        p.calcBlockID()
        p.calcForce()
        if mode == "bucket":
            check_cells(p, s, po)
        got.append({f: p.get(f) for f in ("pid", "cell_start", "r_sorted", "F")})
        p.close()
    for f in got[0]:
        assert np.array_equal(got[0][f], got[1][f]), f


def test_force_c1_vs_oracle_and_reference(cuda_lib, po, golden):
    s = W.config_c1()
    s.r = golden["c1_r4"][:, :3].astype(np.float64)
    p = md(cuda_lib, s)
    p.calcBlockID()
    p.calcForce(energy=True)
    F = p.get("F")
    assert np.all(F[:, 3] == 0)
    Fo, info = oracle_forces(po, s)
    assert relrms(F[:, :3].astype(np.float64), Fo) < FORCE_RELRMS
    sums = p.sums()
    O = po.Oracle(s.box, s.lj, s.rc, s.r)
    e = O.forces()
    assert sums["pe"] == pytest.approx(e["pe"], rel=1e-6)
    assert sums["pe_shift"] == pytest.approx(e["pe_shift"], rel=1e-6)
    assert sums["virial"] == pytest.approx(e["virial"], rel=1e-6)
    # closer to FP64 than the reference's own FP32 kernel
    Fr = golden["c1_F"][:, :3].astype(np.float64)
    assert relrms(F[:, :3].astype(np.float64), Fo) < relrms(Fr, Fo)


def test_force_fp64_accumulation(cuda_lib, po, golden):
    s = W.config_c1()
    s.r = golden["c1_r4"][:, :3].astype(np.float64)
    p = md(cuda_lib, s, fp64_forces=True)
    p.calcBlockID()
    p.calcForce()
    Fo, _ = oracle_forces(po, s)
    assert relrms(p.get("F")[:, :3].astype(np.float64), Fo) < FORCE_RELRMS


def test_force_1m_vs_oracle(cuda_lib, po):
    s = perturbed(W.config_c2(), 0.08, 3)
    p = md(cuda_lib, s, gaussian=True)
    p.calcBlockID()
    p.calcForce(energy=True)
    F = p.get("F")[:, :3].astype(np.float64)
    Fo, info = oracle_forces(po, s)
    assert relrms(F, Fo) < FORCE_RELRMS
    assert p.sums()["pe"] == pytest.approx(
        po.Oracle(s.box, s.lj, s.rc, s.r.astype(np.float32).astype(np.float64)).forces()["pe"],
        rel=1e-6)


def test_force_kob_andersen_per_pair_cutoff(cuda_lib, po):
    s = W.kob_andersen_random(6000, 1.2, 0.8, seed=4)
    O = po.Oracle(s.box, s.lj, s.rc, s.r, s.v, types=s.types)
    O.steepest_descent(60, 1e-3, 0.02)
    s.r = O.get("r").astype(np.float32).astype(np.float64)
    p = md(cuda_lib, s)
    p.calcBlockID()
    p.calcForce()
    Fo, _ = oracle_forces(po, s)
    assert relrms(p.get("F")[:, :3].astype(np.float64), Fo) < FORCE_RELRMS


def test_vv_matches_reference_kernels(cuda_lib, golden):
    s = W.config_c1()
    s.r = golden["c1_r4"][:, :3].astype(np.float64)
    s.v = golden["c1_v"].astype(np.float64)
    p = md(cuda_lib, s)
    p.clearForce()
    for _ in range(10):
        p.calcBlockID()
        p.calcForce()
        p.TimeEvolution(0.005)
        p.treatPeriodicCondition()
    L = float(s.box[1])
    d = p.get("r")[:, :3] - golden["c1_vv10_r4"][:, :3]
    d -= L * np.round(d / L)
    assert np.abs(d).max() < 2e-5
    assert np.abs(p.get("v")[:, :3] - golden["c1_vv10_v4"][:, :3]).max() < 2e-4


def test_gaussian_matches_reference_kernels(cuda_lib, golden):
    s = W.config_c1()
    s.r = golden["c1_r4"][:, :3].astype(np.float64)
    s.v = golden["c1_v"].astype(np.float64)
    p = md(cuda_lib, s, gaussian=True)
    p.clearForce()
    p.run(0.005, 10)
    L = float(s.box[1])
    d = p.get("r")[:, :3] - golden["c1_gauss10_r4"][:, :3]
    d -= L * np.round(d / L)
    assert np.abs(d).max() < 2e-5
    assert np.abs(p.get("vd") - golden["c1_gauss10_vd"]).max() < 2e-4
    assert p.sums()["xi"] == pytest.approx(float(golden["c1_gauss10_xi"][0]), rel=1e-5)


def test_gaussian_fp32_velocities(cuda_lib, po):
    s = W.config_c1()
    p = md(cuda_lib, s, gaussian=True, fp64_velocities=False)
    p.clearForce()
    p.run(0.005, 20)
    O = po.Oracle(s.box, s.lj, s.rc, s.r.astype(np.float32).astype(np.float64),
                  s.v.astype(np.float32).astype(np.float64))
    O.set_tol(1e-12)
    O.run(20, 0.005, mode="gauss")
    L = float(s.box[1])
    d = p.get("r")[:, :3] - O.get("r")
    d -= L * np.round(d / L)
    assert np.abs(d).max() < 1e-4
    assert p.sums()["xi"] == pytest.approx(O.xi, rel=1e-4)


def test_graph_run_equals_eager_steps(cuda_lib):
    s = W.config_c1()
    a = md(cuda_lib, s)
    b = md(cuda_lib, s)
    a.clearForce()
    b.clearForce()
    a.run(0.005, 20)
    for _ in range(20):
        b.calcBlockID()
        b.calcForce()
        b.TimeEvolution(0.005)
        b.treatPeriodicCondition()
    assert np.array_equal(a.get("r"), b.get("r"))
    assert np.array_equal(a.get("v"), b.get("v"))


@pytest.mark.parametrize("gaussian", [False, True])
def test_temperature_after_steps_reuses_the_step_sum(cuda_lib, gaussian):
    """calcTemp after a step reads the sum m v^2 that the step's last kernel computed;
    it must equal the sum recomputed from the same velocities, bit for bit."""
    s = W.config_c1()
    p = md(cuda_lib, s, gaussian=gaussian)
    p.clearForce()
    for steps in (1, 2, 5):
        p.run(0.005, steps)
        t_step = p.calcTemp()           # the step's own sum
        field = "vd" if gaussian else "v"
        p.set(field, p.get(field))      # same velocities: the next read recomputes the sum
        t_fresh = p.calcTemp()
        assert t_step == t_fresh
        # the value is the kinetic temperature of the velocities on the host
        v = p.velocities()
        t_host = float((s.mass[:, None] * v * v).sum()) / (3 * s.n)
        assert t_step == pytest.approx(t_host, rel=1e-6)


def test_deterministic(cuda_lib):
    s = W.config_c1()
    out = []
    for _ in range(2):
        p = md(cuda_lib, s, gaussian=True)
        p.clearForce()
        p.run(0.005, 50)
        out.append((p.get("r"), p.get("vd"), p.sums()["xi"]))
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
    assert out[0][2] == out[1][2]


def test_wrap_bit_exact(cuda_lib, golden):
    box = golden["wrap_box"]
    win = golden["wrap_in"]
    s = W.LJSystem(box=box, r=win[:, :3].astype(np.float64), v=np.zeros((len(win), 3)),
                   mass=np.ones(len(win)), types=np.zeros(len(win), np.uint32),
                   lj=W.single_type_lj(), rc=2.5)
    p = md(cuda_lib, s)
    p.treatPeriodicCondition()
    assert np.array_equal(p.get("r")[:, :3], golden["wrap_out"][:, :3])


def nve_energies(p, steps, dt):
    e = []
    p.clearForce()
    for _ in range(steps):
        p.calcBlockID()
        p.calcForce(energy=True)
        pe = p.sums()["pe_shift"]
        p.TimeEvolution(dt)
        p.treatPeriodicCondition()
        e.append(0.5 * p.sums()["mv2"] + pe)
    return np.array(e) / p.n


def test_nve_drift_c1(cuda_lib):
    s = W.config_c1()
    p = md(cuda_lib, s)
    e = nve_energies(p, 1000, 0.005)[1:]
    drift = np.polyfit(np.arange(len(e)), e, 1)[0] * 1000
    assert abs(drift) < 1e-4, drift
    assert e.std() < 2e-4


def test_small_box_three_cells(cuda_lib, po):
    s = perturbed(W.fcc_system(5, 0.9, 1.0, seed=9), 0.05, 1)  # 500 atoms, 3^3 cells
    p = md(cuda_lib, s)
    assert list(p.grid()[0]) == [3, 3, 3]
    p.calcBlockID()
    check_cells(p, s, po)
    p.calcForce()
    Fo, _ = oracle_forces(po, s)
    assert relrms(p.get("F")[:, :3].astype(np.float64), Fo) < FORCE_RELRMS


def test_two_atoms_analytic_and_across_faces(cuda_lib):
    box = np.array([0, 10, 0, 10, 0, 10], np.float32)
    for d in (0.95, 2 ** (1 / 6), 2.2):
        for axis in range(3):
            for base in (0.3, 5.0):
                r = np.full((2, 3), 5.0)
                r[0, axis] = base
                r[1, axis] = (base - d) % 10.0  # crosses the face when base < d
                s = W.LJSystem(box=box, r=r, v=np.zeros((2, 3)), mass=np.ones(2),
                               types=np.zeros(2, np.uint32), lj=W.single_type_lj(), rc=2.5)
                p = md(cuda_lib, s)
                p.calcBlockID()
                p.calcForce()
                F = p.get("F")
                f = 24 * (2 * d ** -12 - d ** -6) / d
                assert F[0, axis] == pytest.approx(f, rel=2e-5, abs=2e-4)
                assert F[1, axis] == pytest.approx(-f, rel=2e-5, abs=2e-4)


@pytest.mark.parametrize("fp64_sums", [False, True])
def test_open_box_vs_reference_kernels(cuda_lib, golden, fp64_sums):
    """setupCutoffBlock(rmax, periodic = false) against the reference's kernels
    on the same input (golden): the grid with one block past each top face,
    every atom's cell (atoms past the top faces and below the bottom ones
    included), the neighbour table with UINT_MAX outside, and the forces, which
    take no image across a face; a step leaves positions unwrapped."""
    r4 = golden["open_r4"]
    r = r4[:, :3].astype(np.float64)
    box = np.array([0, 20, 0, 20, 0, 20], np.float32)
    s = W.LJSystem(box=box, r=r, v=np.zeros_like(r), mass=np.ones(len(r)),
                   types=np.zeros(len(r), np.uint32), lj=W.single_type_lj(), rc=2.5)
    p = md(cuda_lib, s, fp64_forces=fp64_sums)
    p.setupCutoffBlock(2.5, periodic=False)
    n3, ln, C = p.grid()
    assert np.array_equal(n3, golden["open_grid"]) and np.all(ln == np.float32(2.5))
    p.calcBlockID()
    assert np.array_equal(p.get("cell_of"), golden["open_cell_of"])
    assert np.array_equal(p.get("neighbors"), golden["open_neighbors"])
    p.calcForce()
    F = p.get("F")[:, :3].astype(np.float64)
    assert relrms(F, golden["open_F"][:, :3].astype(np.float64)) < FORCE_RELRMS
    # one velocity-Verlet step: the atoms past the top faces stay there
    p.clearForce()
    p.run(0.001, 1)
    r_after = p.get("r")[:, :3]
    assert r_after[-1].min() > 20.0 and r_after[-2][0] < 0.0
    assert p.status() == 0
    p.close()


def test_open_box_rejects_half_shell_and_lists(cuda_lib, golden):
    r = golden["open_r4"][:, :3].astype(np.float64)
    s = W.LJSystem(box=np.array([0, 20, 0, 20, 0, 20], np.float32), r=r, v=np.zeros_like(r),
                   mass=np.ones(len(r)), types=np.zeros(len(r), np.uint32),
                   lj=W.single_type_lj(), rc=2.5)
    from particlebase_b200._lib import PBError
    p = md(cuda_lib, s, half_shell=True)
    with pytest.raises(PBError):
        p.setupCutoffBlock(2.5, periodic=False)
    p.close()
    q = md(cuda_lib, s)
    q.setupCutoffBlock(2.5, periodic=False)
    with pytest.raises(PBError):
        q.useNList(0.3)
    q.close()


def test_empty_cells_and_crowded_cells(cuda_lib, po):
    """Sparse gas with many empty cells plus a clump of 60 atoms in one cell:
    exercises empty ranges, the >32-member cell ordering and the global-memory
    fallback of the force kernel when its shared-memory stage overflows."""
    rng = np.random.default_rng(2)
    L = 30.0
    gas = rng.uniform(0, L, (800, 3))
    clump = 15.0 + rng.uniform(0, 2.4, (60, 3))
    r = np.concatenate([gas, clump])
    box = np.array([0, L, 0, L, 0, L], np.float32)
    s = W.LJSystem(box=box, r=r, v=np.zeros_like(r), mass=np.ones(len(r)),
                   types=np.zeros(len(r), np.uint32), lj=W.single_type_lj(), rc=2.5)
    p = md(cuda_lib, s)
    p.calcBlockID()
    check_cells(p, s, po)
    p.calcForce()
    Fo, _ = oracle_forces(po, s)
    assert relrms(p.get("F")[:, :3].astype(np.float64), Fo) < FORCE_RELRMS


def test_smem_overflow_fallback(cuda_lib, po):
    """A dense ball far above the mean occupancy overflows the staged capacity;
    the kernel switches to global loads, flags it, and stays correct."""
    rng = np.random.default_rng(4)
    L = 40.0
    gas = rng.uniform(0, L, (2000, 3))
    ball = 20.0 + rng.normal(0, 1.5, (3000, 3))
    r = np.mod(np.concatenate([gas, ball]), L)
    box = np.array([0, L, 0, L, 0, L], np.float32)
    s = W.LJSystem(box=box, r=r, v=np.zeros_like(r), mass=np.ones(len(r)),
                   types=np.zeros(len(r), np.uint32), lj=W.single_type_lj(), rc=2.5)
    p = md(cuda_lib, s)
    p.status()
    p.calcBlockID()
    p.calcForce()
    assert p.status() & 1  # kStatusSmemOverflow
    Fo, _ = oracle_forces(po, s)
    F = p.get("F")[:, :3].astype(np.float64)
    assert relrms(F, Fo) < FORCE_RELRMS


def test_status_clean_after_normal_run(cuda_lib):
    p = md(cuda_lib, W.config_c1(), gaussian=True)
    p.clearForce()
    p.run(0.005, 10)
    assert p.status() == 0


def test_errors_are_returned_not_fatal(cuda_lib):
    from particlebase_b200 import _lib as L
    from particlebase_b200.md import MDSystem
    p = MDSystem(100)
    with pytest.raises(L.PBError) as e:
        p.calcForce()
    assert e.value.code == 3  # PB_ERR_STATE
    p.setCell([0, 5, 0, 5, 0, 5])
    with pytest.raises(L.PBError) as e:
        p.setupCutoffBlock(2.5)  # 2 cells per axis: the reference asserts blocknum > 2
    assert e.value.code == 1
    # an open box has one cell past each top face: 5 / 3 -> 1 + 1 = 2 cells, too few
    with pytest.raises(L.PBError) as e:
        p.setupCutoffBlock(3.0, periodic=False)
    assert e.value.code == 1
    p.setupCutoffBlock(2.5, periodic=False)  # 2 + 1 = 3 cells per axis
    assert list(p.grid()[0]) == [3, 3, 3]


def test_minimize_matches_oracle(cuda_lib, po):
    """Capped steepest descent (extension) on the GPU follows the oracle's
    relaxation from a random Kob-Andersen start, and removes the overlaps."""
    s = W.kob_andersen_random(4000, 1.2, 0.8, seed=6)
    s.r = s.r.astype(np.float32).astype(np.float64)
    p = md(cuda_lib, s)
    O = po.Oracle(s.box, s.lj, s.rc, s.r, s.v, types=s.types)
    p.minimize(10, 1e-3, 0.02)
    O.steepest_descent(10, 1e-3, 0.02)
    d = p.get("r")[:, :3].astype(np.float64) - O.get("r")
    d -= np.round(d / s.L) * s.L
    assert np.abs(d).max() < 1e-3
    p.minimize(190, 1e-3, 0.02)
    p.calcBlockID()
    p.calcForce(energy=True)
    assert p.status() == 0
    assert p.sums()["pe"] / s.n < -4.0  # the random start is far above zero


@pytest.mark.parametrize("gaussian", [False, True])
def test_runs_of_odd_length_match_one_run(cuda_lib, gaussian):
    """Whole steps replay from CUDA graphs that bake in which force buffer is
    F and which is Fold; runs of odd length flip that parity, and later runs
    must still pick the graph captured at the current parity.  Pieces of
    1, 2, 3 and 4 steps give the same bits as one run of 10."""
    from particlebase_b200.md import from_system
    s = perturbed(W.fcc_system(6, 0.8442, 0.72, seed=61), 0.05, 62)
    a = from_system(s, gaussian=gaussian)
    a.clearForce()
    for k in (1, 2, 3, 4):
        a.run(0.005, k)
    b = from_system(s, gaussian=gaussian)
    b.clearForce()
    b.run(0.005, 10)
    assert np.array_equal(a.get("r"), b.get("r"))
    assert np.array_equal(a.get("F"), b.get("F"))


def test_wait_timeout_is_reported_and_the_handle_recovers(cuda_lib, po):
    """Failure detection without a GPU fault: a test hook makes the force
    kernel's producer warps withhold their first hand-off, so the consumer
    warps' bounded wait (2,000 polls of at most 1 us) runs out.  The call
    returns, PB_STATUS_WAIT_TIMEOUT is set, and the next force call on the
    same handle is complete and correct."""
    s = perturbed(W.config_c1(), 0.05, 3)
    p = md(cuda_lib, s)
    p.calcBlockID()
    assert p.status() == 0
    p.force_wait_test(2000)
    assert p.status() & 0x4, "PB_STATUS_WAIT_TIMEOUT"
    p.calcForce()
    assert p.status() == 0
    Fo, _ = oracle_forces(po, s, p.get("r"))
    assert relrms(p.get("F")[:, :3].astype(np.float64), Fo) < FORCE_RELRMS
