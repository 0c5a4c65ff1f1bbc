"""Velocity initialisation, rescaling and the soft-core annealing stage on the
GPU (through the C ABI), against golden vectors of the reference's own kernels
(tests/golden/make_golden.py items 10-12):

* adjustVelocities: adjustVelocity_F4 / adjustVelocity_VD (kernelfuncs.cu:546-699),
  cudaParticleMD.cu:177-198, GaussianThermo.cu:98-119;
* scaleTemp: mulArray (kerneltemplate.hh:29-35) with the factor of
  cudaParticleMD.cu:168-175 and GaussianThermo.cu:89-96;
* initialAnnealing (cudaParticleMD.cu:205-325): the soft-core force
  MDpairForce<potentialSC> (kerneltemplate.hh:523-565, kernelinline.hh:136-158),
  constTemp's correctConstTemp_F4 (kernelfuncs.cu:533-544), the Euler step
  calcA_F4 + propagateEuler_F4 (kernelfuncs.cu:70-82, 174-192), and the whole
  two-stage sequence.
"""
import numpy as np
import pytest

from particlebase_b200 import workloads as W

pytestmark = pytest.mark.gpu


def relrms(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


def c1_handle(golden, v, **kw):
    from particlebase_b200.md import from_system
    s = W.config_c1()
    s.r = golden["c1_r4"][:, :3].astype(np.float64)
    s.v = np.asarray(v, np.float64)
    return from_system(s, **kw), s


def interior_mask(golden):
    L = float(golden["c1_box"][1])
    x = golden["c1_r4"][:, :3]
    return np.all((x > 2.5) & (x < L - 2.5), axis=1)


def test_adjust_velocities_fp32(cuda_lib, golden):
    p, s = c1_handle(golden, golden["vel_in"])
    p.adjustVelocities(float(golden["vel_v1_T"][1]))
    v = p.get("v")[:, :3]
    ref = golden["adjust_vv_v4"][:, :3]
    # (v - mean) * v1 / sqrt(var) in FP64, rounded once to FP32: equal up to
    # one rounding step where the FP64 sums differ in their last bits
    assert np.abs(v - ref).max() <= 2.0 ** -22 * np.abs(ref).max()
    assert (v == ref).mean() > 0.99


def test_adjust_velocities_fp64(cuda_lib, golden):
    p, s = c1_handle(golden, golden["vel_in"], gaussian=True)
    p.adjustVelocities(float(golden["vel_v1_T"][1]))
    assert np.abs(p.get("vd") - golden["adjust_gauss_vd"]).max() < 1e-13


def test_scale_temp_fp32(cuda_lib, golden):
    p, s = c1_handle(golden, golden["vel_in"])
    f = p.scaleTemp(1.1)
    # T0 comes from an FP64 sum here and from a sequential FP32 dot product of
    # 16,000 terms in the reference (its cublasSdot), good to about 1e-6
    assert f == pytest.approx(golden["scale_factors"][0], rel=1e-6)
    assert np.allclose(p.get("v")[:, :3], golden["scale_vv_v4"][:, :3], rtol=1e-6, atol=1e-7)


def test_scale_temp_fp64(cuda_lib, golden):
    p, s = c1_handle(golden, golden["vel_in"], gaussian=True)
    f = p.scaleTemp(1.1)
    assert f == pytest.approx(golden["scale_factors"][1], rel=1e-7)
    assert np.allclose(p.get("vd"), golden["scale_gauss_vd"], rtol=1e-7, atol=1e-9)


def test_softcore_force_consttemp_and_euler(cuda_lib, golden):
    rc, f0, dt = golden["sc_rc_f0_dt"]
    p, s = c1_handle(golden, golden["c1_v"])
    p.calcBlockID()
    p.calcForceSoftCore(float(rc), float(f0))
    F = p.get("F")[:, :3].astype(np.float64)
    ref = golden["sc_F"][:, :3].astype(np.float64)
    inner = interior_mask(golden)
    # FP32 rounding away from the faces; near them the reference's minimum
    # image in r^2 (kernelinline.hh:47-62) costs it two digits, this path uses
    # exact frame shifts
    assert relrms(F[inner], ref[inner]) < 2e-6
    assert relrms(F, ref) < 2e-4
    p.constTemp()
    Fc = p.get("F")[:, :3].astype(np.float64)
    assert relrms(Fc, golden["sc_F_corrected"][:, :3].astype(np.float64)) < 2e-4
    p.stepEuler(float(dt))
    L = float(s.box[1])
    d = p.get("r")[:, :3] - golden["sc_euler_r4"][:, :3]
    d -= L * np.round(d / L)
    assert np.abs(d).max() < 1e-5
    assert np.abs(p.get("v")[:, :3] - golden["sc_euler_v4"][:, :3]).max() < 1e-6


def test_initial_annealing(cuda_lib, golden):
    steps, dt, rc, f0, T = golden["anneal_args"]
    p, s = c1_handle(golden, golden["c1_v"])
    p.initialAnnealing(int(steps), float(dt), float(rc), float(f0), float(T))
    L = float(s.box[1])
    d = p.get("r")[:, :3] - golden["anneal_r4"][:, :3]
    d -= L * np.round(d / L)
    assert np.abs(d).max() < 2e-5
    assert np.abs(p.get("v")[:, :3] - golden["anneal_v4"][:, :3]).max() < 2e-4
    assert p.status() == 0
