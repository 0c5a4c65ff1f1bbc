"""Generate golden vectors from the reference's own MD kernels.

The reference (particlelover/ParticleBase) ships no unit tests or fixtures.
This script runs its kernels -- compiled for the CPU into oracle/_ref by
oracle/Makefile (calcBID_F4, the sortByBID family, makeBindex,
calc_BlockNeighbor, calcF_IJpairWithBlock_F4<MDpairForce<potentialLJ>> +
reduce27_F4, propagateVelocityVerlet_F4, the Gaussian-thermostat kernels,
applyPeriodicCondition_F4, adjustVelocity_F4 / adjustVelocity_VD, mulArray
(scaleTemp), MDpairForce<potentialSC>, correctConstTemp_F4, calcA_F4 and
propagateEuler_F4 of initialAnnealing; the open-box grid and block neighbours of
setupCutoffBlock(rmax, false)) -- on small seeded inputs and stores the outputs in
tests/golden/*.npz.  The oracle is checked against these files in
tests/test_oracle.py, so the pin holds where the reference checkout is absent.

    python tests/golden/make_golden.py      # needs oracle/_ref (make -C oracle ref)
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import pyoracle as po  # noqa: E402
from particlebase_b200 import workloads as W  # noqa: E402


def perturbed_c1(seed: int = 11, amp: float = 0.06):
    s = W.config_c1(seed=1)
    rng = np.random.default_rng(seed)
    r = s.r + rng.uniform(-amp, amp, s.r.shape)
    L = float(s.box[1])
    r = np.mod(r, L)
    r = np.minimum(r.astype(np.float32), np.nextafter(np.float32(L), np.float32(0)))
    return s, r.astype(np.float64)


def ref_system(s, r, gaussian=False, tol=1e-8):
    return po.RefKernels(s.box, s.rc, r, s.v, s.mass, s.types, [1.0, 1.0], gaussian=gaussian,
                         tol=tol)


def main() -> None:
    po.build(ref=True)
    if not po.ref_available():
        raise SystemExit("oracle/_ref is not built (needs the reference checkout)")
    out = {}

    # 1. cell table of C1 (4,000 fcc atoms, 6^3 cells), perturbed positions
    s, r = perturbed_c1()
    R = ref_system(s, r)
    R.calc_block_id()
    bid, pid, bindex = R.cells()
    cell_of = np.empty(s.n, np.uint32)
    cell_of[pid] = bid
    n3, blocklen = R.grid()
    out.update(c1_box=s.box, c1_r4=R.get4("r"), c1_cell_of=cell_of, c1_blocknum=n3,
               c1_blocklen=blocklen[:3], c1_neighbors=R.neighbors(),
               c1_v=s.v.astype(np.float32))

    # 2. forces of the same snapshot (FP32 reference kernel)
    R.calc_force()
    out["c1_F"] = R.get4("F")

    # 3. 10 velocity-Verlet steps (calcBlockID, calcForce, TimeEvolution, wrap)
    R2 = ref_system(s, r)
    R2.run(0.005, 10)
    out["c1_vv10_r4"] = R2.get4("r")
    out["c1_vv10_v4"] = R2.get4("v")

    # 4. 10 Gaussian-thermostat steps at the reference's default Newton-Raphson
    # tolerance (GaussianThermo() : _e(1e-8)).  With 1e-10, as testMD2 sets,
    # the FP32/FP64 mix of the reference kernels stalls at step 9 of this run
    # and the reference would exit(0) (GaussianThermo.cu:42-45).
    R3 = ref_system(s, r, gaussian=True)
    if R3.run(0.005, 10) < 0:
        raise SystemExit("reference Newton-Raphson did not converge")
    out["c1_gauss10_r4"] = R3.get4("r")
    out["c1_gauss10_vd"] = R3.vd()
    out["c1_gauss10_xi"] = np.array([R3.xi])

    # 5. two-body forces in a 10 x 10 x 10 box along x, y and z.  The first
    # atom sits in cell 0: makeBindex sets bindex[0] = 0 unconditionally
    # (kernelfuncs.cu:896), so with cell 0 empty the reference would file the
    # first occupied cell's atoms under cell 0 (see item 8).
    dists = np.array([0.9, 2 ** (1 / 6), 1.5, 2.49, 2.51], np.float64)
    box = np.array([0, 10, 0, 10, 0, 10], np.float32)
    pair_F = []
    for d in dists:
        for axis in range(3):
            rr = np.full((2, 3), 0.5)
            rr[1, axis] += d
            Rp = po.RefKernels(box, 2.5, rr, np.zeros((2, 3)), np.ones(2), np.zeros(2, np.uint32),
                               [1.0, 1.0])
            Rp.calc_block_id()
            Rp.calc_force()
            pair_F.append(Rp.get4("F"))
    out["pair_dist"] = dists
    out["pair_F"] = np.stack(pair_F)

    # 6. minimum image across each face: a pair straddling x, y, z = 0
    img_F = []
    for axis in range(3):
        rr = np.full((2, 3), 0.3)
        rr[1, axis] = 9.5   # nearest image of atom 1 is at -0.5: distance 0.8
        Rp = po.RefKernels(box, 2.5, rr, np.zeros((2, 3)), np.ones(2), np.zeros(2, np.uint32),
                           [1.0, 1.0])
        Rp.calc_block_id()
        Rp.calc_force()
        img_F.append(Rp.get4("F"))
    out["image_F"] = np.stack(img_F)

    # 7. periodic wrap of out-of-box FP32 coordinates
    rng = np.random.default_rng(5)
    rw = rng.uniform(-25.0, 35.0, (256, 3))
    Rw = po.RefKernels(box, 2.5, rw, np.zeros((256, 3)), np.ones(256), np.zeros(256, np.uint32),
                       [1.0, 1.0])
    out["wrap_box"] = box
    out["wrap_in"] = Rw.get4("r")
    Rw.wrap()
    out["wrap_out"] = Rw.get4("r")

    # 8. the makeBindex quirk itself: the same pair as item 6 (x axis) moved to
    # y = z = 5 leaves cell 0 empty; the reference then returns zero force.
    rr = np.full((2, 3), 5.0)
    rr[0, 0] = 0.3
    rr[1, 0] = 9.5
    Rq = po.RefKernels(box, 2.5, rr, np.zeros((2, 3)), np.ones(2), np.zeros(2, np.uint32),
                       [1.0, 1.0])
    Rq.calc_block_id()
    Rq.calc_force()
    out["quirk_r"] = rr
    out["quirk_F"] = Rq.get4("F")

    # 9. g(r): pair counts per bin from the reference's calcF_IJpairWithBlock5_F4
    # with calcGR_F4 (cudaCalcGR), 500 fcc atoms perturbed by 0.2 sigma, bins of
    # 0.05 sigma up to 4 sigma (just under half the 8.4-sigma box)
    sg = W.fcc_system(5, 0.8442, 0.72, seed=3)
    rng = np.random.default_rng(4)
    rg = np.mod(sg.r + rng.uniform(-0.2, 0.2, sg.r.shape), sg.L).astype(np.float32).astype(
        np.float64)
    Rg = ref_system(sg, rg)
    Rg.calc_block_id()
    out["gr_box"] = sg.box
    out["gr_r4"] = Rg.get4("r")
    out["gr_rstep_rmax"] = np.array([0.05, 4.0], np.float32)
    out["gr_counts"] = Rg.gr_counts(0.05, 4.0)

    # 10. velocity initialisation and rescaling (adjustVelocity_F4 / _VD,
    # scaleTemp with mulArray) on 4,000 atoms whose velocities have a nonzero
    # mean and unequal spreads per axis.  v1 = sqrt(kB T / m0) in FP32, T 0.72.
    rng = np.random.default_rng(21)
    v_raw = rng.normal([0.3, -0.2, 0.1], [1.0, 0.7, 1.3], (s.n, 3)).astype(np.float32)
    v1 = float(np.sqrt(np.float32(1.0) * np.float32(0.72) / np.float32(1.0), dtype=np.float32))
    out["vel_in"] = v_raw
    out["vel_v1_T"] = np.array([v1, 0.72], np.float64)
    Ra = po.RefKernels(s.box, s.rc, r, v_raw.astype(np.float64), s.mass, s.types, [1.0, 1.0])
    Ra.adjust_velocities(v1)
    out["adjust_vv_v4"] = Ra.get4("v")
    Rb = po.RefKernels(s.box, s.rc, r, v_raw.astype(np.float64), s.mass, s.types, [1.0, 1.0],
                       gaussian=True)
    Rb.adjust_velocities(v1)
    out["adjust_gauss_vd"] = Rb.vd()
    # scaleTemp to T = 1.1 from the raw velocities
    Rc = po.RefKernels(s.box, s.rc, r, v_raw.astype(np.float64), s.mass, s.types, [1.0, 1.0])
    fvv = Rc.scale_temp(1.1)
    out["scale_vv_v4"] = Rc.get4("v")
    Rd = po.RefKernels(s.box, s.rc, r, v_raw.astype(np.float64), s.mass, s.types, [1.0, 1.0],
                       gaussian=True)
    fg = Rd.scale_temp(1.1)
    out["scale_gauss_vd"] = Rd.vd()
    out["scale_factors"] = np.array([fvv, fg], np.float64)

    # 11. initialAnnealing's pieces on the perturbed C1 snapshot with the
    # MB velocities: the soft-core force (range 1.2, strength 1.0), constTemp's
    # correction of it, and one Euler step (dt 0.005) with the corrected force.
    Rs = ref_system(s, r)
    Rs.calc_block_id()
    Rs.calc_force_softcore(1.2, 1.0)
    out["sc_rc_f0_dt"] = np.array([1.2, 1.0, 0.005], np.float64)
    out["sc_F"] = Rs.get4("F")
    t_ct, lam = Rs.const_temp()
    out["sc_consttemp_T_lambda"] = np.array([t_ct, lam], np.float64)
    out["sc_F_corrected"] = Rs.get4("F")
    Rs.euler(0.005)
    out["sc_euler_r4"] = Rs.get4("r")
    out["sc_euler_v4"] = Rs.get4("v")

    # 12. a short initialAnnealing: 5 soft-core Euler steps with the range
    # growing to 1.2 (f0 1.0, dt 0.005), rescale to T 0.72, 5 LJ VV steps with
    # constTemp, rescale.
    Rn = ref_system(s, r)
    Rn.initial_annealing(5, 0.005, 1.2, 1.0, 0.72)
    out["anneal_args"] = np.array([5, 0.005, 1.2, 1.0, 0.72], np.float64)
    out["anneal_r4"] = Rn.get4("r")
    out["anneal_v4"] = Rn.get4("v")

    # 13. open boundaries (setupCutoffBlock(rmax, periodic = false)): a jittered
    # simple-cubic gas in a 20-sigma box, plus atoms in the extra block past
    # the top faces and just below the bottom ones (clamped to cell 0).
    rng = np.random.default_rng(13)
    g = (np.arange(12) + 0.5) * (20.0 / 12)
    ro = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    ro = ro + rng.uniform(-0.2, 0.2, ro.shape)
    extra = np.array([[20.6, 10.0, 10.0], [10.0, 21.2, 5.0], [3.0, 3.0, 21.9],
                      [-0.05, 12.0, 12.0], [21.5, 21.5, 21.5]])
    ro = np.concatenate([ro, extra]).astype(np.float32).astype(np.float64)
    so = W.LJSystem(box=np.array([0, 20, 0, 20, 0, 20], np.float32), r=ro,
                    v=np.zeros_like(ro), mass=np.ones(len(ro)),
                    types=np.zeros(len(ro), np.uint32), lj=W.single_type_lj(), rc=2.5)
    Ro = po.RefKernels(so.box, so.rc, ro, so.v, so.mass, so.types, [1.0, 1.0], periodic=False)
    Ro.calc_block_id()
    bid, pid, _ = Ro.cells()
    cell_of = np.empty(so.n, np.uint32)
    cell_of[pid] = bid
    Ro.calc_force()
    out["open_r4"] = Ro.get4("r")
    out["open_grid"] = Ro.grid()[0]
    out["open_cell_of"] = cell_of
    out["open_neighbors"] = Ro.neighbors()
    out["open_F"] = Ro.get4("F")

    path = os.path.join(HERE, "reference_kernels.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
