"""Pins of the FP64 oracle (CPU only).

The reference has no tests or fixtures of its own, so the oracle is pinned
two ways: against golden vectors produced by the reference's own kernels
(tests/golden/reference_kernels.npz, made by tests/golden/make_golden.py from
oracle/_ref), and, where the reference checkout is present, against those
kernels directly on further inputs.  Plus known answers: analytic two-body
forces, the zero net force of a perfect fcc lattice, momentum conservation.
"""
import numpy as np
import pytest

from particlebase_b200 import workloads as W


def relrms(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


def lj_force_analytic(r, sigma=1.0, eps=1.0):
    return 24 * eps * (2 * (sigma / r) ** 12 - (sigma / r) ** 6) / r


def test_grid_matches_reference(po, golden):
    n, ln = po.grid(golden["c1_box"], 2.5)
    assert np.array_equal(n, golden["c1_blocknum"])
    assert np.array_equal(ln, golden["c1_blocklen"])  # bit-exact FP32 blocklen


def test_cell_of_matches_reference(po, golden):
    cid = po.bin_cells(golden["c1_r4"], golden["c1_box"], 2.5)
    assert np.array_equal(cid, golden["c1_cell_of"])


def test_neighbor_table_matches_reference(po, golden):
    assert np.array_equal(po.neighbor_table(golden["c1_box"], 2.5), golden["c1_neighbors"])


OPEN_BOX = np.array([0, 20, 0, 20, 0, 20], np.float32)


def open_box_direct_forces(r4, rc=2.5):
    """Truncated LJ (sigma = eps = 1) summed over all pairs, no images (FP64)."""
    r = r4[:, :3].astype(np.float64)
    F = np.zeros_like(r)
    for i in range(len(r)):
        d = r[i] - r
        r2 = (d * d).sum(1)
        m = (r2 < rc * rc) & (r2 > 0)
        inv2 = 1.0 / r2[m]
        s6 = inv2 ** 3
        F[i] = ((24.0 * s6 * (2.0 * s6 - 1.0) * inv2)[:, None] * d[m]).sum(0)
    return F


def test_open_box_cells_match_reference(po, golden):
    """setupCutoffBlock(rmax, periodic = false): one block of length rmax past
    each top face, no wrapped neighbours (UINT_MAX), and the same clamps."""
    n, ln = po.grid(OPEN_BOX, 2.5, periodic=False)
    assert np.array_equal(n, golden["open_grid"])
    assert np.all(ln == np.float32(2.5))
    assert np.array_equal(po.bin_cells(golden["open_r4"], OPEN_BOX, 2.5, periodic=False),
                          golden["open_cell_of"])
    assert np.array_equal(po.neighbor_table(OPEN_BOX, 2.5, periodic=False),
                          golden["open_neighbors"])


def test_open_box_forces_match_reference(golden):
    """The reference's force kernels on the open box equal the all-pairs sum
    without images (the pins the GPU's open-box forces are checked against)."""
    F = open_box_direct_forces(golden["open_r4"])
    assert relrms(golden["open_F"][:, :3].astype(np.float64), F) < 1e-6


def test_cell_list_is_stable_counting_sort(po):
    rng = np.random.default_rng(0)
    cid = rng.integers(0, 50, 1000).astype(np.uint32)
    start, members = po.cell_list(cid, 50)
    assert start[-1] == 1000
    for c in range(50):
        m = members[start[c]:start[c + 1]]
        assert np.all(cid[m] == c)
        assert np.all(np.diff(m.astype(np.int64)) > 0)  # ascending particle id


def test_cell_list_orders_by_z_then_id(po):
    rng = np.random.default_rng(1)
    cid = rng.integers(0, 20, 2000).astype(np.uint32)
    z = rng.integers(0, 30, 2000).astype(np.float32) * np.float32(0.25)  # many ties
    start, members = po.cell_list(cid, 20, z)
    for c in range(20):
        m = members[start[c]:start[c + 1]]
        assert np.all(cid[m] == c)
        key = list(zip(z[m].tolist(), m.tolist()))
        assert key == sorted(key)


def test_forces_match_reference_kernel(po, golden):
    r4 = golden["c1_r4"]
    O = po.Oracle(golden["c1_box"], W.single_type_lj(), 2.5, r4[:, :3].astype(np.float64))
    info = O.forces()
    F = O.get("F")
    Fr = golden["c1_F"][:, :3].astype(np.float64)
    L = float(golden["c1_box"][1])
    x = r4[:, :3]
    interior = np.all((x > 2.5) & (x < L - 2.5), axis=1)
    # Away from the faces the FP32 reference kernel and the FP64 oracle agree to
    # FP32 rounding.  Near the faces the reference's minimum image in r^2,
    # dx^2 + 4 (c - sqrt(c dx^2)) (kernelinline.hh:47-62), cancels and costs it
    # about two decimal digits, hence the looser whole-system bound.
    assert relrms(Fr[interior], F[interior]) < 2e-6
    assert relrms(Fr, F) < 1e-4
    assert info["ncand"] == 4000 * (27 * 4000 / 216 - 1)
    assert np.abs(F.sum(0)).max() < 1e-9  # Newton's third law in aggregate


def test_pair_forces_analytic_and_reference(po, golden):
    box = np.array([0, 10, 0, 10, 0, 10], np.float32)
    k = 0
    for d in golden["pair_dist"]:
        for axis in range(3):
            rr = np.full((2, 3), 0.5)
            rr[1, axis] += d
            O = po.Oracle(box, W.single_type_lj(), 2.5, rr)
            O.forces()
            F = O.get("F")
            expect = lj_force_analytic(d) if d < 2.5 else 0.0
            assert F[0, axis] == pytest.approx(-expect, rel=1e-12, abs=1e-15)
            assert F[1, axis] == pytest.approx(expect, rel=1e-12, abs=1e-15)
            Fr = golden["pair_F"][k][:, :3]
            # FP32 reference: at the force minimum r = 2^(1/6) the factor
            # 2 (s/r)^6 - 1 cancels, so the absolute bound is on the force
            # scale 24 eps / sigma.
            assert np.allclose(F, Fr, rtol=2e-6, atol=24 * 2e-6)
            k += 1


def test_minimum_image_across_faces(po, golden):
    box = np.array([0, 10, 0, 10, 0, 10], np.float32)
    for axis in range(3):
        rr = np.full((2, 3), 0.3)
        rr[1, axis] = 9.5
        O = po.Oracle(box, W.single_type_lj(), 2.5, rr)
        O.forces()
        F = O.get("F")
        f = lj_force_analytic(0.8)
        assert F[0, axis] == pytest.approx(f, rel=1e-12)  # pushed away from the image at -0.5
        # FP32 reference through its sqrt-based image distance: ~1e-4 relative
        assert np.allclose(F, golden["image_F"][axis][:, :3], rtol=3e-4)


def test_reference_empty_cell0_quirk_is_not_reproduced(po, golden):
    """makeBindex writes bindex[0] = 0 unconditionally (kernelfuncs.cu:896):
    with cell 0 empty the reference misfiles the first occupied cell and this
    pair gets no force.  The oracle (and the CUDA path) use correct cell ranges."""
    assert np.all(golden["quirk_F"][:, :3] == 0)
    box = np.array([0, 10, 0, 10, 0, 10], np.float32)
    O = po.Oracle(box, W.single_type_lj(), 2.5, golden["quirk_r"])
    O.forces()
    assert O.get("F")[0, 0] == pytest.approx(lj_force_analytic(0.8), rel=1e-12)


def test_wrap_bit_exact_with_reference(po, golden):
    w = po.wrap_f32(golden["wrap_in"], golden["wrap_box"])
    assert np.array_equal(w[:, :3], golden["wrap_out"][:, :3])


def test_vv_trajectory_matches_reference(po, golden):
    r4 = golden["c1_r4"]
    box = golden["c1_box"]
    L = float(box[1])
    O = po.Oracle(box, W.single_type_lj(), 2.5, r4[:, :3].astype(np.float64),
                  golden["c1_v"].astype(np.float64))
    O.run(10, 0.005)
    d = O.get("r") - golden["c1_vv10_r4"][:, :3]
    d -= L * np.round(d / L)
    assert np.abs(d).max() < 2e-5
    assert np.abs(O.get("v") - golden["c1_vv10_v4"][:, :3]).max() < 2e-4


def test_gaussian_trajectory_matches_reference(po, golden):
    r4 = golden["c1_r4"]
    box = golden["c1_box"]
    L = float(box[1])
    O = po.Oracle(box, W.single_type_lj(), 2.5, r4[:, :3].astype(np.float64),
                  golden["c1_v"].astype(np.float64))
    O.set_tol(1e-8)
    O.run(10, 0.005, mode="gauss")
    d = O.get("r") - golden["c1_gauss10_r4"][:, :3]
    d -= L * np.round(d / L)
    assert np.abs(d).max() < 2e-5
    assert np.abs(O.get("v") - golden["c1_gauss10_vd"]).max() < 2e-4
    assert O.xi == pytest.approx(float(golden["c1_gauss10_xi"][0]), rel=1e-5)


def test_gaussian_holds_kinetic_energy(po):
    # The discrete isokinetic scheme of GaussianThermo keeps sum m v^2 to
    # O(dt^2) per step, not exactly; the reference kernels show the same drift.
    s = W.config_c1()
    O = po.Oracle(s.box, s.lj, s.rc, s.r, s.v)
    O.set_tol(1e-12)
    k0 = O.kinetic()
    O.run(20, 0.005, mode="gauss")
    assert O.kinetic() == pytest.approx(k0, rel=5e-3)


def test_gaussian_closed_form_equals_newton_raphson(po):
    """xi = c / (1 - c dt/2) with c = sum F.A / sum m A^2 is the fixed point
    the reference's Newton-Raphson loop converges to (GaussianThermo.cu:29-77)."""
    s = W.config_c1()
    dt = 0.005
    O = po.Oracle(s.box, s.lj, s.rc, s.r, s.v)
    O.set_tol(1e-13)
    O.run(3, dt, mode="gauss")  # arbitrary state with nonzero Fold, xi
    v0, xi0, fold = O.get("v"), O.xi, O.get("Fold")
    O.forces()
    F = O.get("F")
    A = v0 + (F + fold) * dt / 2 - v0 * xi0 * dt / 2
    c = (F * A).sum() / (A * A).sum()
    xi = c / (1 - c * dt / 2)
    O.run(1, dt, mode="gauss")
    assert O.xi == pytest.approx(xi, rel=1e-10)
    assert np.allclose(O.get("v"), A / (1 + xi * dt / 2), rtol=1e-10, atol=1e-12)


def test_gaussian_first_step_stops_after_one_iteration(po):
    """With xi(t-dt) = 0 the reference's initial guess v = A satisfies its
    convergence test at once: v = A and xi = sum F.A / sum m A^2."""
    s = W.config_c1()
    dt = 0.005
    O = po.Oracle(s.box, s.lj, s.rc, s.r, s.v)
    O.set_tol(1e-13)
    O.forces()
    F = O.get("F")
    A = s.v + F * dt / 2
    O.run(1, dt, mode="gauss")
    assert O.xi == pytest.approx((F * A).sum() / (A * A).sum(), rel=1e-12)
    assert np.allclose(O.get("v"), A, rtol=1e-12, atol=1e-14)


def test_fcc_lattice_has_zero_force(po):
    s = W.fcc_system(6, 0.8442, 0.0 + 1e-9, seed=0)
    O = po.Oracle(s.box, s.lj, s.rc, s.r)
    O.forces()
    assert np.abs(O.get("F")).max() < 1e-10


def test_nve_conserves_shifted_energy(po):
    # Truncated-force dynamics conserve KE + sum (U(r) - U(rc)); the first step
    # is skipped because Fold = 0 there (cudaParticleVV::clearForce) gives the
    # reference scheme a one-off double force kick.
    s = W.config_c1()
    O = po.Oracle(s.box, s.lj, s.rc, s.r, s.v)
    e = O.run(400, 0.005, record=True)[1:]
    etot = (e[:, 0] + e[:, 2]) / s.n
    drift = np.polyfit(np.arange(len(etot)), etot, 1)[0] * 1000
    assert abs(drift) < 1e-4
    assert np.std(etot) < 2e-4


@pytest.mark.skipif("not __import__('pyoracle').ref_available()")
def test_kob_andersen_forces_vs_reference_kernel(po):
    """Two-type system with one global cutoff (the reference has no per-pair rc)."""
    s = W.kob_andersen_random(3000, 1.2, 0.8, seed=3)
    O = po.Oracle(s.box, s.lj, s.rc, s.r, s.v, types=s.types)
    O.steepest_descent(30, 1e-3, 0.02)
    r = O.get("r")
    lj_global = s.lj.copy()
    lj_global[..., 2] = 2.5
    O2 = po.Oracle(s.box, lj_global, 2.5, r.astype(np.float32).astype(np.float64), types=s.types)
    O2.forces()
    R = po.RefKernels(s.box, 2.5, r, s.v, s.mass, s.types, s.lj[..., :2].reshape(-1), ntypes=2)
    R.calc_block_id()
    R.calc_force()
    F = O2.get("F")
    Fr = R.get4("F")[:, :3].astype(np.float64)
    assert relrms(Fr, F) < 2e-4


def test_gr_counts_match_reference_kernel(po, golden):
    """The oracle's g(r) pair counts equal those of the reference's own
    calcF_IJpairWithBlock5_F4 / calcGR_F4 kernel (golden fixture) bin for bin."""
    rstep, rmax = (float(x) for x in golden["gr_rstep_rmax"])
    counts = po.gr_counts(golden["gr_r4"], golden["gr_box"], rstep, rmax)
    assert np.array_equal(counts, golden["gr_counts"].astype(np.int64))
    n = len(golden["gr_r4"])
    L = golden["gr_box"][1] - golden["gr_box"][0]
    g = po.gr_normalise(counts, n, float(L) ** 3, rstep)
    assert g[0] == 0 and g.max() > 1.5  # the perturbed lattice's first shell


# ---- velocity initialisation, rescaling and the annealing stage ---------------
# Golden items 10-12 of tests/golden/make_golden.py: adjustVelocity_F4 /
# adjustVelocity_VD, scaleTemp (mulArray), the soft-core force of
# initialAnnealing (MDpairForce<potentialSC>), constTemp's correction
# (correctConstTemp_F4), the Euler step (calcA_F4 + propagateEuler_F4) and a
# short initialAnnealing, all from the reference's own kernels.

def _c1_oracle(golden, v=None):
    r4 = golden["c1_r4"]
    return po_oracle(golden, r4, v)


def po_oracle(golden, r4, v):
    import pyoracle
    return pyoracle.Oracle(golden["c1_box"], W.single_type_lj(), 2.5,
                           r4[:, :3].astype(np.float64),
                           None if v is None else np.asarray(v, np.float64))


def test_adjust_velocities_matches_reference(po, golden):
    v1 = float(golden["vel_v1_T"][0])
    O = _c1_oracle(golden, golden["vel_in"])
    O.adjust_velocities(v1)
    v = O.get("v")
    # FP32 velocities of adjustVelocity_F4: (v - mean) * v1 rsqrt(var) in FP64,
    # rounded once to FP32
    assert np.abs(v - golden["adjust_vv_v4"][:, :3]).max() <= 4e-7 * np.abs(v).max()
    # adjustVelocity_VD keeps FP64: agreement to FP64 summation order
    assert np.abs(v - golden["adjust_gauss_vd"]).max() < 1e-13
    assert np.abs(v.mean(0)).max() < 1e-12
    assert np.allclose(v.std(0), v1, rtol=1e-12)


def test_scale_temp_matches_reference(po, golden):
    O = _c1_oracle(golden, golden["vel_in"])
    f = O.scale_temp(1.1)
    fvv, fg = golden["scale_factors"]
    # GaussianThermo::scaleTemp takes T0 from calcTemp() as `real` (FP32), then
    # an FP64 square root; cudaParticleMD::scaleTemp is FP32 throughout
    assert f == pytest.approx(fg, rel=1e-7)
    assert f == pytest.approx(fvv, rel=1e-6)
    assert np.allclose(O.get("v"), golden["scale_gauss_vd"], rtol=1e-7, atol=1e-9)
    assert np.allclose(O.get("v"), golden["scale_vv_v4"][:, :3], rtol=1e-6, atol=1e-7)


def test_softcore_force_and_euler_match_reference(po, golden):
    rc, f0, dt = golden["sc_rc_f0_dt"]
    O = _c1_oracle(golden, golden["c1_v"])
    O.forces_softcore(rc, f0)
    F = O.get("F")
    Fr = golden["sc_F"][:, :3].astype(np.float64)
    L = float(golden["c1_box"][1])
    x = golden["c1_r4"][:, :3]
    interior = np.all((x > 2.5) & (x < L - 2.5), axis=1)
    # as for the LJ force: FP32 rounding away from the faces, the reference's
    # minimum image in r^2 near them
    assert relrms(Fr[interior], F[interior]) < 2e-6
    assert relrms(Fr, F) < 2e-4
    assert np.abs(F.sum(0)).max() < 1e-10  # pairwise and antisymmetric
    lam = O.const_temp()
    T_ref, lam_ref = golden["sc_consttemp_T_lambda"]
    assert lam == pytest.approx(lam_ref, rel=1e-4)
    assert relrms(golden["sc_F_corrected"][:, :3].astype(np.float64), O.get("F")) < 2e-4
    O.euler(dt)
    d = O.get("r") - golden["sc_euler_r4"][:, :3]
    d -= L * np.round(d / L)
    assert np.abs(d).max() < 1e-5
    assert np.abs(O.get("v") - golden["sc_euler_v4"][:, :3]).max() < 1e-6


def test_softcore_force_is_zero_beyond_its_range(po):
    box = np.array([0, 10, 0, 10, 0, 10], np.float32)
    for d, expect in ((0.6, 1.0 * np.cos(0.6 / 1.2 * np.pi / 2)), (1.3, 0.0)):
        rr = np.full((2, 3), 0.5)
        rr[1, 0] += d
        O = po.Oracle(box, W.single_type_lj(), 2.5, rr)
        O.forces_softcore(1.2, 1.0)
        F = O.get("F")
        assert F[0, 0] == pytest.approx(-expect, abs=1e-15)
        assert F[1, 0] == pytest.approx(expect, abs=1e-15)


def test_initial_annealing_matches_reference(po, golden):
    steps, dt, rc, f0, T = golden["anneal_args"]
    O = _c1_oracle(golden, golden["c1_v"])
    O.initial_annealing(int(steps), dt, rc, f0, T)
    L = float(golden["c1_box"][1])
    d = O.get("r") - golden["anneal_r4"][:, :3]
    d -= L * np.round(d / L)
    assert np.abs(d).max() < 2e-5
    assert np.abs(O.get("v") - golden["anneal_v4"][:, :3]).max() < 2e-4
    # the final rescale sets T = 0.72 exactly (up to the (3N - 1) / 3N factor)
    ke = O.kinetic()
    n = len(golden["c1_r4"])
    assert 2 * ke / (3 * n) == pytest.approx(T * (3 * n - 1) / (3 * n), rel=1e-12)
