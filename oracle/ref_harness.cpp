// Host driver for the reference's own MD kernels, compiled for the CPU.
//
// TEST INFRASTRUCTURE ONLY (oracle).  Built by oracle/Makefile into
// oracle/_ref/libpbref.so from the reference sources where they lie; the
// reference files are never copied into this repository.  The build includes
//   kernelfuncs.cu       (calcBID_F4, sortByBID_M1, sortByBID, makeBindex,
//                         reduce27_F4, propagateVelocityVerlet_F4,
//                         applyPeriodicCondition_F4, the Gaussian-thermostat
//                         kernels, calcMV2_F4, calcV2_F4, calcReciproc)
//   kerneltemplate.hh    (clearArray, mulArray, accumulate,
//                         calcF_IJpairWithBlock_F4, MDpairForce)
//   kernelinline.hh      (distance2p, potentialLJ, _setLJparams)
// plus two kernels cut out at build time from files whose host code uses
// <<<>>> launches (calc_BlockNeighbor from cudaCutoffBlock.cu:17-65,
// copyWithIndex from cudaSortedPositions.cu:19-25).
//
// What is written here is only the host-side orchestration, restating the
// reference classes' call order:
//   cudaCutoffBlock::setupCutoffBlock  cudaCutoffBlock.cu:75-231
//   cudaCutoffBlock::calcBlockID       cudaCutoffBlock.cu:233-258
//   cudaSortedPositions::calcBlockID   cudaSortedPositions.cu:27-30
//   cudaParticleMD::calcForce          cudaParticleMD.cu:24-69
//   cudaParticleVV::TimeEvolution      cudaParticleVV.cu:17-34
//   GaussianThermo::TimeEvolution      GaussianThermo.cu:29-77
//   cudaParticleBase::treatPeriodicCondition cudaParticleBase.cu:175-184
// Launch shapes follow CUDAenv<T>::setThnum (CUDAenv.hh:36-50) on a B200 with
// the THnum2D override the reference needs on compute capability 10.x
// (numberOfCores() returns 0 there): MPnum=148, THnum1D=1024, THnum2D=32,
// threadsMax=1024.
//
// One deliberate deviation: innerProduct_F4 (kernelfuncs.cu:473-500) stores
// only the last grid-stride term of each thread (tmp_d[thID] = d), which is
// wrong whenever N exceeds the thread count.  The driver below computes the
// same quantity, sum F.vd in FP64, with a full loop instead.
#include "ref_emu.h"

thread_local uint3 threadIdx;
thread_local uint3 blockIdx;
thread_local dim3 blockDim;
thread_local dim3 gridDim;

// kernelfuncs.cu and kerneltemplate.hh both declare a dynamic shared array
// named tmp_s with different element types; give the first one its own name.
#define tmp_s tmp_s_kernelfuncs
#include "kernelfuncs.cu"
#undef tmp_s
#include "kerneltemplate.hh"
#include "calc_BlockNeighbor.inc"
#include "copyWithIndex.inc"

// Backing storage for the reference's dynamic shared arrays.  Kernels that
// use them run as one single-thread block (never in parallel), so each array
// holds a single partial sum.
double tmp_d[64];
double tmp_v[64 * 6];
real tmp_r[64];
uint32_t tmp_s_kernelfuncs[64];
double tmp_s4[64];
uint32_t subarray[64];
double tmp_s[64];
uint2 red[64 * 64];

#include <omp.h>

namespace {

// Run kernel(args...) as a grid of one-thread blocks.  `parallel` lets
// OpenMP run blocks concurrently; callers set it only for kernels whose
// blocks write disjoint outputs.
template <typename K, typename... A>
void launch(dim3 grid, bool parallel, K kernel, A... args) {
  const long nx = grid.x, ny = grid.y;
#pragma omp parallel for collapse(2) schedule(static) if (parallel)
  for (long y = 0; y < ny; ++y) {
    for (long x = 0; x < nx; ++x) {
      gridDim = grid;
      blockDim = dim3(1, 1, 1);
      threadIdx = uint3{0, 0, 0};
      blockIdx = uint3{(uint32_t)x, (uint32_t)y, 0};
      kernel(args...);
    }
  }
}

struct RefSys {
  uint32_t N = 0;
  bool gaussian = false;
  real cell[9];
  real rmax2 = 0;
  real kB = 1;
  double xi = 0;
  real e = 1e-8f;
  // B200 launch parameters (see file comment)
  int MPnum = 148, THnum1D = 1024, THnum2D = 32;
  uint32_t threadsMax = 1024;
  uint32_t THnum2D2 = 32;
  std::vector<float4> r, v, a, F, tmp3N, r_s;
  std::vector<real> minv, m;
  std::vector<unsigned short> typeID, typeID_s;
  std::vector<uint32_t> bid, pid, bindex, blockNeighbor;
  std::vector<real> tmp81N;
  std::vector<double> vd;
  std::vector<real> blocklen;
  std::vector<uint32_t> blocknum;
  uint32_t totalNumBlock = 0;
  int nr_last = 0;
};

uint32_t threads1D(const RefSys &s) { return (uint32_t)s.MPnum * (uint32_t)s.THnum1D; }

}  // namespace

extern "C" {

void *ref_create(uint32_t N, const float *cell6, int gaussian) {
  RefSys *s = new RefSys;
  s->N = N;
  s->gaussian = gaussian != 0;
  // cudaFrame::setCell, cudaFrame.cu:85-91
  for (int i = 0; i < 6; ++i) s->cell[i] = cell6[i];
  for (int i = 0; i < 3; ++i) {
    s->cell[i + 6] = (s->cell[i * 2 + 1] - s->cell[i * 2]) / 2;
    s->cell[i + 6] *= s->cell[i + 6];
  }
  const float4 z4{0, 0, 0, 0};
  s->r.assign(N, z4);
  s->v.assign(N, z4);
  s->a.assign(N, z4);
  s->F.assign(N, z4);
  s->tmp3N.assign(N, z4);
  s->r_s.assign(N, z4);
  s->minv.assign(N, 0);
  s->m.assign(N, 0);
  s->typeID.assign(N, 0);
  s->typeID_s.assign(N, 0);
  s->vd.assign((size_t)N * 3, 0.0);
  return s;
}

void ref_destroy(void *h) { delete (RefSys *)h; }

void ref_set_rmax2(void *h, float rmax2) { ((RefSys *)h)->rmax2 = rmax2; }
void ref_set_kB(void *h, float kB) { ((RefSys *)h)->kB = kB; }
void ref_set_e(void *h, float e) { ((RefSys *)h)->e = e; }

// _setLJparams (kernelinline.hh:120-134): (sigma, epsilon) per type pair.
void ref_set_lj(void *h, const float *p, uint32_t elemnum) {
  (void)h;
  std::vector<real> P(p, p + 2 * elemnum * elemnum);
  _setLJparams(P, elemnum);
}

// cudaParticleBase::import (cudaParticleBase.cu:68-117), GaussianThermo::import
// (GaussianThermo.cu:16-28) and cudaParticleMD::setM (cudaParticleMD.cu:135-138).
void ref_import(void *h, const double *r3, const double *v3, const double *mass,
                const uint32_t *type) {
  RefSys &s = *(RefSys *)h;
  for (uint32_t i = 0; i < s.N; ++i) {
    s.r[i] = float4{(real)r3[3 * i], (real)r3[3 * i + 1], (real)r3[3 * i + 2], 0};
    s.v[i] = float4{(real)v3[3 * i], (real)v3[3 * i + 1], (real)v3[3 * i + 2], 0};
    s.a[i] = float4{0, 0, 0, 0};
    s.minv[i] = (real)(1.0 / mass[i]);
    s.typeID[i] = (unsigned short)type[i];
    s.vd[i] = v3[3 * i];
    s.vd[i + s.N] = v3[3 * i + 1];
    s.vd[i + 2 * s.N] = v3[3 * i + 2];
  }
  launch(dim3(threads1D(s)), true, calcReciproc, s.minv.data(), s.m.data(), s.N);
}

void ref_set_positions(void *h, const float *r4) {
  RefSys &s = *(RefSys *)h;
  std::memcpy(s.r.data(), r4, sizeof(float4) * s.N);
}

// cudaCutoffBlock::setupCutoffBlock (cudaCutoffBlock.cu:75-231), many-particle
// blocks; periodic, or open (one block of length rmax past each top face, no
// wrapped neighbours).
int ref_setup_cells_p(void *h, float rmax, int periodic) {
  RefSys &s = *(RefSys *)h;
  s.blocklen.assign(6, 0);
  s.blocknum.assign(3, 0);
  s.bid.assign(s.N, 0);
  s.pid.resize(s.N);
  for (uint32_t i = 0; i < s.N; ++i) s.pid[i] = i;
  real c[3];
  for (int i = 0; i < 3; ++i) {
    c[i] = s.cell[i * 2 + 1] - s.cell[i * 2];
    if (periodic) {
      s.blocknum[i] = static_cast<uint32_t>(c[i] / rmax);
      s.blocklen[i] = c[i] / static_cast<real>(s.blocknum[i]);
    } else {
      s.blocklen[i] = rmax;
      s.blocknum[i] = static_cast<uint32_t>(c[i] / rmax) + 1;
    }
    if (s.blocknum[i] <= 2) return -1;
    s.blocklen[i + 3] = s.cell[i * 2];
  }
  s.totalNumBlock = s.blocknum[0] * s.blocknum[1] * s.blocknum[2];
  s.bindex.assign(s.totalNumBlock + 1, 0);
  s.bindex[s.totalNumBlock] = s.N;
  s.blockNeighbor.assign((size_t)s.totalNumBlock * 27, 0);
  launch(dim3(s.MPnum), true, calc_BlockNeighbor, s.blockNeighbor.data(), 1, periodic != 0, 27,
         s.blocknum[0], s.blocknum[1], s.blocknum[2]);
  s.tmp81N.assign((size_t)s.N * 81, 0);
  s.THnum2D2 = s.THnum2D;
  {
    int _N = (real)(s.N) / s.totalNumBlock;
    while ((int)s.THnum2D2 < _N) s.THnum2D2 *= 2;
  }
  return 0;
}

int ref_setup_cells(void *h, float rmax) { return ref_setup_cells_p(h, rmax, 1); }

// cudaCutoffBlock::calcBlockID + cudaSortedPositions::calcBlockID
void ref_calc_block_id(void *h) {
  RefSys &s = *(RefSys *)h;
  const uint32_t T = threads1D(s);
  launch(dim3(T), true, calcBID_F4, s.r.data(), s.bid.data(), s.pid.data(), s.N,
         s.totalNumBlock, s.blocklen[0], s.blocklen[1], s.blocklen[2], s.blocklen[3],
         s.blocklen[4], s.blocklen[5], s.blocknum[0], s.blocknum[1], s.blocknum[2]);
  launch(dim3(T), true, clearArray<uint32_t>, s.bindex.data(), s.totalNumBlock,
         (uint32_t)UINT_MAX);
  int M1 = s.MPnum;
  int T1 = s.THnum2D;
  while ((M1 * T1 > 32) && (M1 > 1) && (T1 > 1)) {
    launch(dim3((uint32_t)(M1 * T1)), true, sortByBID_M1, s.pid.data(), s.bid.data(), s.N);
    if ((T1 * 2) > M1) {
      T1 /= 2;
    } else {
      M1 /= 2;
    }
  }
  launch(dim3(1), false, sortByBID, s.pid.data(), s.bid.data(), s.N);
  launch(dim3(T), true, makeBindex, s.bid.data(), s.bindex.data(), s.N);
  launch(dim3(T), true, copyWithIndex<float4>, s.r.data(), s.r_s.data(), s.N, s.pid.data());
  launch(dim3(T), true, copyWithIndex<unsigned short>, s.typeID.data(), s.typeID_s.data(),
         s.N, s.pid.data());
}

// cudaParticleMD::calcForce, cell-block branch (cudaParticleMD.cu:24-60).
void ref_calc_force(void *h) {
  RefSys &s = *(RefSys *)h;
  const uint32_t T = threads1D(s);
  launch(dim3(T), true, clearArray_F4, s.F.data(), s.N, float4{0, 0, 0, 0});
  potentialLJ LJ;
  MDpairForce<potentialLJ> P;
  P.cx = s.cell[6];
  P.cy = s.cell[7];
  P.cz = s.cell[8];
  P.c0x = sqrt(P.cx) * 2.0;
  P.c0y = sqrt(P.cy) * 2.0;
  P.c0z = sqrt(P.cz) * 2.0;
  P.rmax2 = s.rmax2;
  P.typeID = s.typeID_s.data();
  P.op = LJ;
  launch(dim3(T), true, clearArray<real>, s.tmp81N.data(), s.N * 81, (real)0);
  // Blocks with different blockIdx.x own different home atoms; blockIdx.y
  // selects a plane, so the whole grid writes disjoint tmp81N entries.
  launch(dim3(s.totalNumBlock, 27), true, calcF_IJpairWithBlock_F4<MDpairForce<potentialLJ>>,
         P, s.r_s.data(), s.tmp81N.data(), (uint32_t)0, s.blockNeighbor.data(), s.pid.data(),
         s.bindex.data(), s.N, (real *)nullptr, (uint32_t *)nullptr, true, false);
  launch(dim3(T), true, reduce27_F4, s.F.data(), s.tmp81N.data(), s.N);
}

// cudaParticleVV::clearForce (cudaParticleVV.cu:10-15); Fold aliases a.
void ref_clear_force(void *h) {
  RefSys &s = *(RefSys *)h;
  const uint32_t T = threads1D(s);
  launch(dim3(T), true, clearArray_F4, s.F.data(), s.N, float4{0, 0, 0, 0});
  launch(dim3(T), true, clearArray_F4, s.a.data(), s.N, float4{0, 0, 0, 0});
}

// GaussianThermo::calcMV2 (GaussianThermo.cu:79-87): FP64 sum, returned as real.
static real gauss_mv2(RefSys &s) {
  const uint32_t T = threads1D(s);
  double *t = reinterpret_cast<double *>(s.tmp3N.data());
  launch(dim3(T), true, calcMV2_F4, s.vd.data(), s.m.data(), t, s.N);
  launch(dim3(1), false, accumulate<double>, t, s.N, t);
  return (real)t[0];
}

// cudaParticleMD::calcMV2 (cudaParticleMD.cu:124-133).  cublasSdot is
// replaced by a sequential FP32 dot product (cuBLAS's order is not public).
static real vv_mv2(RefSys &s) {
  const uint32_t T = threads1D(s);
  float *t = reinterpret_cast<float *>(s.tmp3N.data());
  launch(dim3(T), true, calcV2_F4, s.v.data(), t, s.N);
  float acc = 0;
  for (uint32_t i = 0; i < s.N; ++i) acc += t[i] * s.m[i];
  return acc;
}

double ref_calc_mv2(void *h) {
  RefSys &s = *(RefSys *)h;
  return s.gaussian ? (double)gauss_mv2(s) : (double)vv_mv2(s);
}

// Returns the number of Newton-Raphson iterations (Gaussian) or 0, or -1 when
// the reference loop would have called exit(0) (GaussianThermo.cu:42-45).
int ref_time_evolution(void *h, float dt) {
  RefSys &s = *(RefSys *)h;
  const uint32_t T = threads1D(s);
  if (!s.gaussian) {
    launch(dim3(T), true, propagateVelocityVerlet_F4, s.r.data(), dt, s.v.data(), s.F.data(),
           s.a.data(), s.minv.data(), s.N);
    return 0;
  }
  double *A = reinterpret_cast<double *>(s.tmp81N.data());
  double *t3 = reinterpret_cast<double *>(s.tmp3N.data());
  launch(dim3(T), true, calcGaussianThermoA1_F4, A, dt, s.vd.data(), s.F.data(), s.a.data(),
         s.minv.data(), s.N, s.xi);
  double v0 = 0;
  uint32_t it = 0;
  double mv2inv = 1.0 / gauss_mv2(s);
  do {
    if (it++ > 50) return -1;
    launch(dim3(T), true, calcGaussianThermoFoverF_F4, A, dt, s.vd.data(), s.F.data(),
           s.m.data(), t3, s.N, s.xi, (real)mv2inv);
    launch(dim3(1), false, accumulate<double>, t3, s.N, t3);
    v0 = t3[0];
    v0 = sqrt(v0 / (s.N * 3));
    // innerProduct_F4 replacement: full FP64 sum of F.vd
    double fv = 0;
    for (uint32_t i = 0; i < s.N; ++i) {
      fv += s.F[i].x * s.vd[i];
      fv += s.F[i].y * s.vd[i + s.N];
      fv += s.F[i].z * s.vd[i + 2 * s.N];
    }
    s.xi = fv;
    mv2inv = 1.0 / gauss_mv2(s);
    s.xi *= mv2inv;
  } while (v0 > s.e);
  launch(dim3(T), true, propagateVelocityVerletGaussianThermo_F4, s.r.data(), dt, s.vd.data(),
         s.F.data(), s.a.data(), s.minv.data(), s.N, s.xi);
  s.nr_last = (int)it;
  return (int)it;
}

void ref_wrap(void *h) {
  RefSys &s = *(RefSys *)h;
  float3 c1{s.cell[0], s.cell[2], s.cell[4]};
  float3 c2{s.cell[1], s.cell[3], s.cell[5]};
  launch(dim3(threads1D(s)), true, applyPeriodicCondition_F4, s.r.data(), c1, c2, s.N);
}

// cudaParticleMD::adjustVelocities (cudaParticleMD.cu:177-198) and
// GaussianThermo::adjustVelocities (GaussianThermo.cu:98-119): the reference
// launches adjustVelocity_F4 / adjustVelocity_VD (kernelfuncs.cu:546-699) as
// one block of min(1024, threadsMax) threads.  Here the same kernel runs as
// one thread (st = 1): the per-axis sums are the same FP64 sums added in
// sequence instead of by the block's tree.  v1 is the caller's
// sqrt(kB T / m0) in `real`, as the reference computes it.
void ref_adjust_velocities(void *h, float v1) {
  RefSys &s = *(RefSys *)h;
  if (s.gaussian)
    launch(dim3(1), false, adjustVelocity_VD, s.vd.data(), (uint32_t)1, s.N, (real)v1,
           (float *)nullptr);
  else
    launch(dim3(1), false, adjustVelocity_F4, s.v.data(), (uint32_t)1, s.N, (real)v1,
           (float *)nullptr);
}

// cudaParticleMD::scaleTemp (cudaParticleMD.cu:168-175; FP32 factor, mulArray
// over the 4 N floats of v) and GaussianThermo::scaleTemp (GaussianThermo.cu:89-96;
// FP64 factor over the 3 N doubles of vd).  T0 is calcTemp()
// (cudaParticleMD.hh:89-92) = calcMV2 / (3 N kB).  Returns the factor.
double ref_scale_temp(void *h, float T) {
  RefSys &s = *(RefSys *)h;
  const uint32_t Tn = threads1D(s);
  const real mv2 = s.gaussian ? gauss_mv2(s) : vv_mv2(s);
  const real T0 = mv2 / (s.N * 3 * s.kB);
  if (s.gaussian) {
    const double f = sqrt(static_cast<double>(3 * s.N - 1) / static_cast<double>(3 * s.N) * T / T0);
    launch(dim3(Tn), true, mulArray<double>, s.vd.data(), f, s.N * 3);
    return f;
  }
  const real f = sqrt(static_cast<real>(3 * s.N - 1) / static_cast<real>(3 * s.N) * T / T0);
  launch(dim3(Tn), true, mulArray<float>, reinterpret_cast<float *>(s.v.data()), f, s.N * 4);
  return f;
}

// The soft-core force of initialAnnealing (cudaParticleMD.cu:226-262):
// calcF_IJpairWithBlock_F4<MDpairForce<potentialSC>> (kerneltemplate.hh:229-294,
// 523-565; potentialSC kernelinline.hh:136-158) + reduce27_F4 on the current
// cell list, with P.rmax2 the LJ cutoff and op.rc, op.f0 as given.
void ref_calc_force_softcore(void *h, float rc, float f0) {
  RefSys &s = *(RefSys *)h;
  const uint32_t T = threads1D(s);
  launch(dim3(T), true, clearArray_F4, s.F.data(), s.N, float4{0, 0, 0, 0});
  potentialSC SC;
  SC.rc = rc;
  SC.f0 = f0;
  MDpairForce<potentialSC> P;
  P.cx = s.cell[6];
  P.cy = s.cell[7];
  P.cz = s.cell[8];
  P.c0x = sqrt(P.cx) * 2.0;
  P.c0y = sqrt(P.cy) * 2.0;
  P.c0z = sqrt(P.cz) * 2.0;
  P.rmax2 = s.rmax2;
  P.typeID = s.typeID_s.data();
  P.op = SC;
  launch(dim3(T), true, clearArray<real>, s.tmp81N.data(), s.N * 81, (real)0);
  launch(dim3(s.totalNumBlock, 27), true, calcF_IJpairWithBlock_F4<MDpairForce<potentialSC>>,
         P, s.r_s.data(), s.tmp81N.data(), (uint32_t)0, s.blockNeighbor.data(), s.pid.data(),
         s.bindex.data(), s.N, (real *)nullptr, (uint32_t *)nullptr, true, false);
  launch(dim3(T), true, reduce27_F4, s.F.data(), s.tmp81N.data(), s.N);
}

// cudaParticleMD::constTemp (cudaParticleMD.cu:140-155): lambda = sum F.v /
// sum m v^2 over the 4 N floats (cublasSdot replaced by a sequential FP32
// dot product, as in vv_mv2), then correctConstTemp_F4 (kernelfuncs.cu:533-544)
// when lambda != 0.  Returns the temperature t / (3 N kB); *lambda_out = lambda.
double ref_const_temp(void *h, double *lambda_out) {
  RefSys &s = *(RefSys *)h;
  const real t = vv_mv2(s);
  real lambda = 0;
  const float *F = reinterpret_cast<const float *>(s.F.data());
  const float *v = reinterpret_cast<const float *>(s.v.data());
  for (uint32_t i = 0; i < 4 * s.N; ++i) lambda += F[i] * v[i];
  lambda /= t;
  if (lambda != 0)
    launch(dim3(threads1D(s)), true, correctConstTemp_F4, s.v.data(), s.F.data(), s.m.data(),
           lambda, s.N);
  if (lambda_out) *lambda_out = lambda;
  return t / (3 * s.N * s.kB);
}

// The Euler step of initialAnnealing (cudaParticleMD.cu:271-277): calcA_F4
// (kernelfuncs.cu:70-82) into a, propagateEuler_F4 (kernelfuncs.cu:174-192)
// with every particle movable (move[i] = 1), applyPeriodicCondition_F4.
void ref_euler(void *h, float dt) {
  RefSys &s = *(RefSys *)h;
  const uint32_t T = threads1D(s);
  std::vector<char> move(s.N, 1);
  launch(dim3(T), true, calcA_F4, s.a.data(), s.minv.data(), s.F.data(), s.N);
  launch(dim3(T), true, propagateEuler_F4, s.r.data(), (real)dt, s.v.data(), s.a.data(),
         move.data(), s.N);
  ref_wrap(h);
}

// cudaParticleMD::initialAnnealing (cudaParticleMD.cu:205-325) for the plain
// MD class: anealstep soft-core Euler steps whose range grows to rc, a
// temperature rescale, anealstep LJ velocity-Verlet steps with constTemp, and
// a final rescale.  The second stage clears Fold (cudaParticleMD.cu:289).
void ref_initial_annealing(void *h, uint32_t anealstep, float dt, float rc, float f0, float T) {
  RefSys &s = *(RefSys *)h;
  const uint32_t Tn = threads1D(s);
  for (uint32_t i = 0; i < anealstep; ++i) {
    const real rci = rc * (i + 1) / anealstep;
    ref_calc_block_id(h);
    ref_calc_force_softcore(h, rci, f0);
    ref_const_temp(h, nullptr);
    ref_euler(h, dt);
  }
  ref_scale_temp(h, T);
  launch(dim3(Tn), true, clearArray_F4, s.a.data(), s.N, float4{0, 0, 0, 0});
  for (uint32_t i = 0; i < anealstep; ++i) {
    ref_calc_block_id(h);
    ref_calc_force(h);
    ref_const_temp(h, nullptr);
    launch(dim3(Tn), true, propagateVelocityVerlet_F4, s.r.data(), (real)dt, s.v.data(),
           s.F.data(), s.a.data(), s.minv.data(), s.N);
    ref_wrap(h);
  }
  ref_scale_temp(h, T);
}

void ref_set_v(void *h, const float *v4) {
  RefSys &s = *(RefSys *)h;
  std::memcpy(s.v.data(), v4, sizeof(float4) * s.N);
}

void ref_set_F(void *h, const float *F4) {
  RefSys &s = *(RefSys *)h;
  std::memcpy(s.F.data(), F4, sizeof(float4) * s.N);
}

// Driver order of testMD2.cu:149-168 / testMD1.cu:135-154 without the
// temperature policy: calcBlockID, calcForce, TimeEvolution, PBC.
int ref_run(void *h, float dt, uint32_t steps) {
  int rc = 0;
  for (uint32_t k = 0; k < steps; ++k) {
    ref_calc_block_id(h);
    ref_calc_force(h);
    rc = ref_time_evolution(h, dt);
    if (rc < 0) return rc;
    ref_wrap(h);
  }
  return rc;
}

void ref_get_r(void *h, float *out) {
  RefSys &s = *(RefSys *)h;
  std::memcpy(out, s.r.data(), sizeof(float4) * s.N);
}
void ref_get_v(void *h, float *out) {
  RefSys &s = *(RefSys *)h;
  std::memcpy(out, s.v.data(), sizeof(float4) * s.N);
}
void ref_get_F(void *h, float *out) {
  RefSys &s = *(RefSys *)h;
  std::memcpy(out, s.F.data(), sizeof(float4) * s.N);
}
void ref_get_Fold(void *h, float *out) {
  RefSys &s = *(RefSys *)h;
  std::memcpy(out, s.a.data(), sizeof(float4) * s.N);
}
void ref_get_vd(void *h, double *out) {
  RefSys &s = *(RefSys *)h;
  std::memcpy(out, s.vd.data(), sizeof(double) * 3 * s.N);
}
double ref_get_xi(void *h) { return ((RefSys *)h)->xi; }
uint32_t ref_num_cells(void *h) { return ((RefSys *)h)->totalNumBlock; }
void ref_get_grid(void *h, uint32_t *blocknum3, float *blocklen6) {
  RefSys &s = *(RefSys *)h;
  for (int i = 0; i < 3; ++i) blocknum3[i] = s.blocknum[i];
  for (int i = 0; i < 6; ++i) blocklen6[i] = s.blocklen[i];
}
void ref_get_cells(void *h, uint32_t *bid, uint32_t *pid, uint32_t *bindex) {
  RefSys &s = *(RefSys *)h;
  std::memcpy(bid, s.bid.data(), 4 * s.N);
  std::memcpy(pid, s.pid.data(), 4 * s.N);
  std::memcpy(bindex, s.bindex.data(), 4 * (s.totalNumBlock + 1));
}
void ref_get_neighbors(void *h, uint32_t *out) {
  RefSys &s = *(RefSys *)h;
  std::memcpy(out, s.blockNeighbor.data(), 4 * (size_t)s.totalNumBlock * 27);
}
int ref_threads(void) { return omp_get_max_threads(); }

}  // extern "C"

extern "C" {

// cudaCalcGR (cudaCalcGR.hh:27-40, cudaCalcGR.cu:52-116) on the CPU: the bin
// count rule of setup(), the pair chunks of makePairInfo() (every pair of
// occupied cell blocks I <= J, in chunks of at most 64 atoms), and the
// reference's own calcF_IJpairWithBlock5_F4 kernel with calcGR_F4
// (kerneltemplate.hh:423-512, kernelinline.hh:433-449) run as one block.
// Needs ref_calc_block_id first.  Returns rnum; fills counts[rnum] when
// counts is non-null and ncounts >= rnum (bin 0 holds nothing).
int ref_gr(void *h, float rstep, float rmax, uint32_t *counts, uint32_t ncounts) {
  RefSys &s = *(RefSys *)h;
  const real rstepinv = 1.0 / rstep;
  const uint32_t rnum = static_cast<uint32_t>(rmax * rstepinv);
  if (!counts) return (int)rnum;
  if (ncounts < rnum) return -1;
  std::vector<uint4> info;
  const std::vector<uint32_t> &bi = s.bindex;
  auto block_end = [&](uint32_t I) {
    uint32_t k = I + 1;
    while (bi[k] == UINT_MAX) ++k;
    return bi[k];
  };
  for (uint32_t I = 0; I < s.totalNumBlock; ++I) {
    if (bi[I] == UINT_MAX) continue;
    const uint32_t i0 = bi[I], i1 = block_end(I);
    for (uint32_t J = I; J < s.totalNumBlock; ++J) {
      if (bi[J] == UINT_MAX) continue;
      const uint32_t j0 = bi[J], j1 = block_end(J);
      for (uint32_t i = i0; i < i1; i += 64)
        for (uint32_t j = j0; j < j1; j += 64)
          info.push_back(uint4{i, std::min(i + 64, i1), j, std::min(j + 64, j1)});
    }
  }
  calcGR_F4 P;
  P.cx = s.cell[6];
  P.cy = s.cell[7];
  P.cz = s.cell[8];
  P.rstepinv = rstepinv;
  P.rnum = rnum;
  P.typeID = nullptr;
  std::vector<uint32_t> igr(rnum, 0);
  launch(dim3(1), false, calcF_IJpairWithBlock5_F4<calcGR_F4>, P, s.r_s.data(), info.data(),
         (uint32_t)info.size(), igr.data(), rnum);
  for (uint32_t k = 0; k < rnum; ++k) counts[k] = igr[k];
  return (int)rnum;
}

}  // extern "C"
