// Velocity Verlet, Gaussian isokinetic thermostat, periodic wrap and the
// FP64 reductions around them, for one or many packed systems.
//
//   k_vv        propagateVelocityVerlet_F4 (kernelfuncs.cu:333-367) fused with
//               applyPeriodicCondition_F4 (kernelfuncs.cu:87-139) and the
//               sum m v^2 of calcMV2 (cudaParticleMD.cu:124-133, FP64 here
//               instead of cublasSdot in FP32).
//   k_gauss_a   first half of GaussianThermo::TimeEvolution
//               (GaussianThermo.cu:29-77): A = v + (F + Fold) dt/2m
//               - v xi(t-dt) dt/2 and the sums F.A, m A^2.
//   k_gauss_b   v = A / (1 + xi dt/2), r += v (dt - xi dt^2/2) + F dt^2/2m,
//               wrap, sum m v^2.
//
// The reference solves v = A - v xi(v) dt/2 with xi(v) = sum F.v / sum m v^2
// by a Newton-Raphson loop that synchronises with the host every iteration.
// For a given xi the equation is linear in each component,
// v = A / (1 + xi dt/2); substituting into xi(v) gives
// xi = c (1 + xi dt/2) with c = sum F.A / sum m A^2, so
// xi = c / (1 - c dt/2).  This is the fixed point the reference iterates
// towards (it stops within its tolerance of it), computed on the device in
// two passes with no host round trip.
//
// One case differs: the reference tests convergence with the xi of the
// previous iteration, and when xi(t-dt) is exactly 0 (the first step after
// construction) its initial guess v = A already gives f = 0, so the loop ends
// after one pass with v = A and xi = sum F.A / sum m A^2 = c.  That step is
// reproduced as the reference computes it.
#include "integrate.cuh"

namespace pb {
namespace {

// Per-system "last block finishes the sum": block b (block k of system s,
// whose blocks are blk0 .. blk0 + nblk - 1) writes its NV partials; the
// system's last block adds the system's partials in block order.  Returns
// true in thread 0 of that block, with the totals in `tot`.
template <int NV>
__device__ __forceinline__ bool sys_total(const double (&mine)[NV], double *partials, uint32_t b,
                                          uint32_t blk0, uint32_t nblk, unsigned int *counter,
                                          double (&tot)[NV], double *scratch) {
  __shared__ bool is_last;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) partials[(size_t)b * NV + k] = mine[k];
    __threadfence();
    const unsigned int ticket = atomicAdd(counter, 1u);
    is_last = (ticket == nblk - 1);
  }
  __syncthreads();
  if (!is_last) return false;
  __threadfence();
  double acc[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k) acc[k] = 0.0;
  for (uint32_t q = threadIdx.x; q < nblk; q += blockDim.x) {
#pragma unroll
    for (int k = 0; k < NV; ++k) acc[k] += __ldcg(&partials[(size_t)(blk0 + q) * NV + k]);
  }
  block_sum<NV>(acc, scratch);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) tot[k] = acc[k];
    *counter = 0;
  }
  return threadIdx.x == 0;
}

__device__ __forceinline__ bool finished(const IntegrateArgs &a, uint32_t sys) {
  return a.steps_left != nullptr && a.steps_left[sys] == 0u;
}

__device__ __forceinline__ void count_step(const IntegrateArgs &a, uint32_t sys) {
  if (a.steps_left != nullptr) a.steps_left[sys] -= 1u;
}

__device__ __forceinline__ void wrap3(const SysInt &S, float4 &p) {
  p.x = wrap_coord(p.x, S.c0[0], S.c1[0], S.L[0]);
  p.y = wrap_coord(p.y, S.c0[1], S.c1[1], S.L[1]);
  p.z = wrap_coord(p.z, S.c0[2], S.c1[2], S.L[2]);
}

// FP64 velocity of atom i (global index) of system S: plane k at vd0 + k * natoms.
__device__ __forceinline__ void load_vd(const IntegrateArgs &a, const SysInt &S, uint32_t i,
                                        double v[3]) {
  const size_t o = (size_t)S.vd0 + (i - S.atom0);
  v[0] = a.vd[o];
  v[1] = a.vd[o + S.natoms];
  v[2] = a.vd[o + 2 * (size_t)S.natoms];
}

__device__ __forceinline__ void store_vd(const IntegrateArgs &a, const SysInt &S, uint32_t i,
                                         const double v[3]) {
  const size_t o = (size_t)S.vd0 + (i - S.atom0);
  a.vd[o] = v[0];
  a.vd[o + S.natoms] = v[1];
  a.vd[o + 2 * (size_t)S.natoms] = v[2];
}

__device__ __forceinline__ void load_v(const IntegrateArgs &a, const SysInt &S, uint32_t i,
                                       double v[3]) {
  if (a.vd) {
    load_vd(a, S, i, v);
  } else {
    const float4 w = a.v[i];
    v[0] = w.x;
    v[1] = w.y;
    v[2] = w.z;
  }
}

__global__ void __launch_bounds__(kIntThreads) k_vv(IntegrateArgs a) {
  pdl_enter();
  __shared__ double red[32];
  const BlockMap m = a.map[blockIdx.x];
  if (finished(a, m.sys)) return;
  const SysInt &S = a.sys[m.sys];
  double mv2 = 0;
  for (uint32_t t = threadIdx.x; t < m.n; t += kIntThreads) {
    const uint32_t i = m.i0 + t;
    const float dt = S.dt;
    const float dt2 = dt * 0.5f;
    const float h = dt2 * a.minv[i];  // dt / 2m
    const float4 F = a.F[i], Fo = a.Fold[i];
    float4 v = a.v[i];
    v.x += (F.x + Fo.x) * h;
    v.y += (F.y + Fo.y) * h;
    v.z += (F.z + Fo.z) * h;
    v.w = 0.f;
    const float h2 = h * dt;
    float4 p = a.r[i];
    p.x += v.x * dt + F.x * h2;
    p.y += v.y * dt + F.y * h2;
    p.z += v.z * dt + F.z * h2;
    if (a.wrap) wrap3(S, p);
    a.v[i] = v;
    a.r[i] = p;
    mv2 += (double)a.mass[i] * ((double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z);
  }
  double s[1] = {mv2}, tot[1];
  block_sum<1>(s, red);
  if (sys_total<1>(s, a.partials, blockIdx.x, S.blk0, S.nblk, &a.sc[m.sys].counter[0], tot, red)) {
    a.sc[m.sys].mv2 = tot[0];
    if (!isfinite(tot[0])) atomicOr(&a.status[m.sys], kStatusNonFinite);
    count_step(a, m.sys);  // every block of the system has read steps_left
  }
}

// Per-atom inputs of the Gaussian passes, read through the read-only data
// path.  A thread's atoms (kIntAtoms / kIntThreads, strided) are taken
// kIntGroup at a time, the loads of a group issued before its arithmetic;
// one atom at a time keeps the register count, and so the number of resident
// threads, highest, which measured fastest.
constexpr int kIntPer = kIntAtoms / kIntThreads;
constexpr int kIntGroup = 1;

struct GaussIn {
  float4 F, Fo;
  double v[3];
  float minv, mass;
};

__device__ __forceinline__ void gauss_load(const IntegrateArgs &a, const SysInt &S, uint32_t i,
                                           GaussIn &g) {
  g.minv = __ldg(a.minv + i);
  g.mass = __ldg(a.mass + i);
  g.F = __ldg(a.F + i);
  g.Fo = __ldg(a.Fold + i);
  load_v(a, S, i, g.v);
}

// A for one atom (FP64), identical arithmetic in both Gaussian passes:
// A = v + (F + Fold) dt/2m - v xi(t-dt) dt/2.
__device__ __forceinline__ void gauss_A(const SysInt &S, const GaussIn &g, double hx,
                                        double A[3]) {
  const float h = (S.dt * 0.5f) * g.minv;
  A[0] = g.v[0] + (double)(g.F.x + g.Fo.x) * h - g.v[0] * hx;
  A[1] = g.v[1] + (double)(g.F.y + g.Fo.y) * h - g.v[1] * hx;
  A[2] = g.v[2] + (double)(g.F.z + g.Fo.z) * h - g.v[2] * hx;
}

// Eight blocks per SM: the first pass fits in 32 registers without spills, and
// the extra resident warps keep more loads in flight (0.040 against 0.043 ms
// for both passes at 1M atoms).  The second pass measured slower when held to
// 40 or 32 registers, which spill.
__global__ void __launch_bounds__(kIntThreads, 8) k_gauss_a(IntegrateArgs a) {
  pdl_enter();
  __shared__ double red[2 * 32];
  const BlockMap m = a.map[blockIdx.x];
  if (finished(a, m.sys)) return;
  const SysInt &S = a.sys[m.sys];
  DevScalars &sc = a.sc[m.sys];
  const double xi_old = sc.xi_old;
  const double hx = (double)S.dt * 0.5 * xi_old;
  double s[2] = {0, 0};
#pragma unroll
  for (int j0 = 0; j0 < kIntPer; j0 += kIntGroup) {
    GaussIn g[kIntGroup];
#pragma unroll
    for (int j = 0; j < kIntGroup; ++j) {
      const uint32_t t = threadIdx.x + (j0 + j) * kIntThreads;
      if (t < m.n) gauss_load(a, S, m.i0 + t, g[j]);
    }
#pragma unroll
    for (int j = 0; j < kIntGroup; ++j) {
      const uint32_t t = threadIdx.x + (j0 + j) * kIntThreads;
      if (t < m.n) {
        double A[3];
        gauss_A(S, g[j], hx, A);
        s[0] += (double)g[j].F.x * A[0] + (double)g[j].F.y * A[1] + (double)g[j].F.z * A[2];
        s[1] += (double)g[j].mass * (A[0] * A[0] + A[1] * A[1] + A[2] * A[2]);
      }
    }
  }
  double tot[2];
  block_sum<2>(s, red);
  if (sys_total<2>(s, a.partials, blockIdx.x, S.blk0, S.nblk, &sc.counter[1], tot, red)) {
    const double hdt = 0.5 * (double)S.dt;
    const double c = tot[1] > 0 ? tot[0] / tot[1] : 0.0;
    double xi = (xi_old == 0.0) ? c : c / (1.0 - c * hdt);
    if (!isfinite(xi) || !isfinite(tot[0]) || !isfinite(tot[1])) {
      atomicOr(&a.status[m.sys], kStatusNonFinite | kStatusNoConverge);
      xi = 0.0;
    }
    sc.sum_fa = tot[0];
    sc.sum_ma2 = tot[1];
    sc.xi_new = xi;
  }
}

__global__ void __launch_bounds__(kIntThreads) k_gauss_b(IntegrateArgs a) {
  pdl_enter();
  __shared__ double red[32];
  const BlockMap m = a.map[blockIdx.x];
  if (finished(a, m.sys)) return;
  const SysInt &S = a.sys[m.sys];
  DevScalars &sc = a.sc[m.sys];
  const double xi_old = sc.xi_old;
  const double xi = sc.xi_new;
  const double hx = (double)S.dt * 0.5 * xi_old;
  const double dt = S.dt;
  const double inv = (xi_old == 0.0) ? 1.0 : 1.0 / (1.0 + xi * 0.5 * dt);
  const double cv = dt - xi * 0.5 * dt * dt;
  double mv2 = 0;
#pragma unroll
  for (int j0 = 0; j0 < kIntPer; j0 += kIntGroup) {
    GaussIn g[kIntGroup];
    float4 p[kIntGroup];
#pragma unroll
    for (int j = 0; j < kIntGroup; ++j) {
      const uint32_t t = threadIdx.x + (j0 + j) * kIntThreads;
      if (t < m.n) {
        gauss_load(a, S, m.i0 + t, g[j]);
        p[j] = a.r[m.i0 + t];
      }
    }
#pragma unroll
    for (int j = 0; j < kIntGroup; ++j) {
      const uint32_t t = threadIdx.x + (j0 + j) * kIntThreads;
      if (t < m.n) {
        const uint32_t i = m.i0 + t;
        double A[3];
        gauss_A(S, g[j], hx, A);
        const double v[3] = {A[0] * inv, A[1] * inv, A[2] * inv};
        const double cf = 0.5 * dt * dt * (double)g[j].minv;
        float4 q = p[j];
        q.x = (float)((double)q.x + v[0] * cv + (double)g[j].F.x * cf);
        q.y = (float)((double)q.y + v[1] * cv + (double)g[j].F.y * cf);
        q.z = (float)((double)q.z + v[2] * cv + (double)g[j].F.z * cf);
        if (a.wrap) wrap3(S, q);
        a.r[i] = q;
        if (a.vd) {
          store_vd(a, S, i, v);
          mv2 += (double)g[j].mass * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        } else {
          const float4 vf = make_float4((float)v[0], (float)v[1], (float)v[2], 0.f);
          a.v[i] = vf;
          mv2 += (double)g[j].mass *
                 ((double)vf.x * vf.x + (double)vf.y * vf.y + (double)vf.z * vf.z);
        }
      }
    }
  }
  double s[1] = {mv2}, tot[1];
  block_sum<1>(s, red);
  if (sys_total<1>(s, a.partials, blockIdx.x, S.blk0, S.nblk, &sc.counter[2], tot, red)) {
    sc.mv2 = tot[0];
    sc.xi_old = xi;  // every other block of this system has finished reading xi_old
    if (!isfinite(tot[0])) atomicOr(&a.status[m.sys], kStatusNonFinite);
    count_step(a, m.sys);
  }
}

__global__ void __launch_bounds__(kIntThreads) k_wrap(IntegrateArgs a) {
  const BlockMap m = a.map[blockIdx.x];
  for (uint32_t t = threadIdx.x; t < m.n; t += kIntThreads) {
    const uint32_t i = m.i0 + t;
    float4 p = a.r[i];
    wrap3(a.sys[m.sys], p);
    a.r[i] = p;
  }
}

__global__ void __launch_bounds__(kIntThreads) k_mv2(IntegrateArgs a) {
  __shared__ double red[32];
  const BlockMap m = a.map[blockIdx.x];
  const SysInt &S = a.sys[m.sys];
  double s[1] = {0};
  for (uint32_t t = threadIdx.x; t < m.n; t += kIntThreads) {
    const uint32_t i = m.i0 + t;
    double v[3];
    load_v(a, S, i, v);
    s[0] += (double)a.mass[i] * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  }
  double tot[1];
  block_sum<1>(s, red);
  if (sys_total<1>(s, a.partials, blockIdx.x, S.blk0, S.nblk, &a.sc[m.sys].counter[0], tot, red))
    a.sc[m.sys].mv2 = tot[0];
}

__global__ void __launch_bounds__(kIntThreads) k_fv(IntegrateArgs a) {
  __shared__ double red[32];
  const BlockMap m = a.map[blockIdx.x];
  const SysInt &S = a.sys[m.sys];
  double s[1] = {0};
  for (uint32_t t = threadIdx.x; t < m.n; t += kIntThreads) {
    const uint32_t i = m.i0 + t;
    const float4 F = a.F[i];
    double v[3];
    load_v(a, S, i, v);
    s[0] += (double)F.x * v[0] + (double)F.y * v[1] + (double)F.z * v[2];
  }
  double tot[1];
  block_sum<1>(s, red);
  if (sys_total<1>(s, a.partials, blockIdx.x, S.blk0, S.nblk, &a.sc[m.sys].counter[3], tot, red))
    a.sc[m.sys].fv = tot[0];
}

__global__ void __launch_bounds__(kIntThreads) k_scale(IntegrateArgs a, const double *f) {
  const BlockMap m = a.map[blockIdx.x];
  for (uint32_t t = threadIdx.x; t < m.n; t += kIntThreads) {
    const SysInt &S = a.sys[m.sys];
    const uint32_t i = m.i0 + t;
    const double s = f[m.sys];
    if (a.vd) {
      double v[3];
      load_vd(a, S, i, v);
      for (int k = 0; k < 3; ++k) v[k] *= s;
      store_vd(a, S, i, v);
    } else {
      const float sf = (float)s;
      float4 v = a.v[i];
      v.x *= sf;
      v.y *= sf;
      v.z *= sf;
      v.w *= sf;
      a.v[i] = v;
    }
  }
}

// adjustVelocity_F4 / adjustVelocity_VD (kernelfuncs.cu:546-699): per axis,
// subtract the mean and scale to standard deviation v1.  Pass 1: sums.
__global__ void __launch_bounds__(kIntThreads) k_vstats(IntegrateArgs a) {
  __shared__ double red[6 * 32];
  const BlockMap m = a.map[blockIdx.x];
  const SysInt &S = a.sys[m.sys];
  double s[6] = {0, 0, 0, 0, 0, 0};
  for (uint32_t t = threadIdx.x; t < m.n; t += kIntThreads) {
    double w[3];
    load_v(a, S, m.i0 + t, w);
    for (int k = 0; k < 3; ++k) {
      s[k] += w[k];
      s[3 + k] += w[k] * w[k];
    }
  }
  double tot[6];
  block_sum<6>(s, red);
  if (sys_total<6>(s, a.partials, blockIdx.x, S.blk0, S.nblk, &a.sc[m.sys].counter[3], tot, red)) {
    for (int k = 0; k < 6; ++k) a.sc[m.sys].vstat[k] = tot[k];
  }
}

__global__ void __launch_bounds__(kIntThreads) k_vapply(IntegrateArgs a, const double *v1s) {
  const BlockMap m = a.map[blockIdx.x];
  for (uint32_t t = threadIdx.x; t < m.n; t += kIntThreads) {
    const SysInt &S = a.sys[m.sys];
    const uint32_t i = m.i0 + t;
    const DevScalars &sc = a.sc[m.sys];
    const double n = (double)S.natoms, v1 = v1s[m.sys];
    double mean[3], f[3];
    for (int k = 0; k < 3; ++k) {
      mean[k] = sc.vstat[k] / n;
      const double var = sc.vstat[3 + k] / n - mean[k] * mean[k];
      f[k] = var > 0 ? v1 / sqrt(var) : 0.0;
    }
    if (a.vd) {
      double v[3];
      load_vd(a, S, i, v);
      for (int k = 0; k < 3; ++k) v[k] = (v[k] - mean[k]) * f[k];
      store_vd(a, S, i, v);
    } else {
      float4 v = a.v[i];
      v.x = (float)((v.x - mean[0]) * f[0]);
      v.y = (float)((v.y - mean[1]) * f[1]);
      v.z = (float)((v.z - mean[2]) * f[2]);
      a.v[i] = v;
    }
  }
}

// calcA_F4 + propagateEuler_F4 + applyPeriodicCondition_F4 of initialAnnealing
// (cudaParticleMD.cu:205-325): r += v dt with the old v, then v += (F/m) dt.
// FP32 velocities only (the annealing belongs to the plain MD class).
__global__ void __launch_bounds__(kIntThreads) k_euler(IntegrateArgs a, const float4 *F, float dt) {
  const BlockMap m = a.map[blockIdx.x];
  for (uint32_t t = threadIdx.x; t < m.n; t += kIntThreads) {
    const SysInt &S = a.sys[m.sys];
    const uint32_t i = m.i0 + t;
    const float mi = a.minv[i];
    const float4 f = F[i];
    float4 v = a.v[i];
    float4 p = a.r[i];
    p.x += v.x * dt;
    p.y += v.y * dt;
    p.z += v.z * dt;
    v.x += f.x * mi * dt;
    v.y += f.y * mi * dt;
    v.z += f.z * mi * dt;
    wrap3(S, p);
    a.v[i] = v;
    a.r[i] = p;
  }
}

// Steepest-descent move (extension, no counterpart in the reference): each
// atom goes along its force by F min(alpha, max_disp / |F|), then wraps.
__global__ void __launch_bounds__(kIntThreads) k_sd_move(IntegrateArgs a, const float4 *F,
                                                        float alpha, float max_disp) {
  const BlockMap m = a.map[blockIdx.x];
  for (uint32_t t = threadIdx.x; t < m.n; t += kIntThreads) {
    const SysInt &S = a.sys[m.sys];
    const uint32_t i = m.i0 + t;
    const float4 f = F[i];
    const float fn = sqrtf(fmaf(f.x, f.x, fmaf(f.y, f.y, f.z * f.z)));
    const float g = fn * alpha > max_disp ? max_disp / fn : alpha;
    float4 p = a.r[i];
    p.x = fmaf(g, f.x, p.x);
    p.y = fmaf(g, f.y, p.y);
    p.z = fmaf(g, f.z, p.z);
    wrap3(S, p);
    a.r[i] = p;
  }
}

// correctConstTemp_F4 (kernelfuncs.cu:533-544): F -= lambda m v, per system.
__global__ void __launch_bounds__(kIntThreads) k_correct(IntegrateArgs a, float4 *F,
                                                        const double *lambda) {
  const BlockMap m = a.map[blockIdx.x];
  for (uint32_t t = threadIdx.x; t < m.n; t += kIntThreads) {
    const SysInt &S = a.sys[m.sys];
    const uint32_t i = m.i0 + t;
    double v[3];
    load_v(a, S, i, v);
    const float l = (float)lambda[m.sys];
    const float mi = a.mass[i];
    float4 f = F[i];
    f.x -= l * mi * (float)v[0];
    f.y -= l * mi * (float)v[1];
    f.z -= l * mi * (float)v[2];
    F[i] = f;
  }
}

// One block per system: energy partials of the system's force items, in order.
__global__ void __launch_bounds__(kIntThreads) k_energy_total(const double *partials,
                                                             const uint32_t *item0,
                                                             DevScalars *sc) {
  __shared__ double red[4 * 32];
  const uint32_t s0 = item0[blockIdx.x], s1 = item0[blockIdx.x + 1];
  double s[4] = {0, 0, 0, 0};
  for (uint32_t b = s0 + threadIdx.x; b < s1; b += blockDim.x) {
    s[0] += partials[(size_t)b * 4 + 0];
    s[1] += partials[(size_t)b * 4 + 1];
    s[2] += partials[(size_t)b * 4 + 2];
    s[3] += partials[(size_t)b * 4 + 3];
  }
  block_sum<4>(s, red);
  if (threadIdx.x == 0) {
    DevScalars &d = sc[blockIdx.x];
    d.pe = s[0];
    d.pe_shift = s[1];
    d.virial = s[2];
    d.npairs = s[3];
  }
}

__global__ void __launch_bounds__(kIntThreads) k_fill_sysid(const BlockMap *map, uint32_t *sysid) {
  const BlockMap m = map[blockIdx.x];
  for (uint32_t t = threadIdx.x; t < m.n; t += kIntThreads) sysid[m.i0 + t] = m.sys;
}

__global__ void __launch_bounds__(kIntThreads) k_gather_state(GatherArgs g) {
  const BlockMap m = g.map[blockIdx.x];
  const GatherSrc q = g.gs[m.sys];
  if (q.src < 0) {  // a new system starts from zeros, as a new engine's arrays do
    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
    for (uint32_t t = threadIdx.x; t < m.n; t += kIntThreads) {
      const uint32_t off = m.k * kIntAtoms + t, i = m.i0 + t;
      g.r[i] = z4;
      g.F0[i] = z4;
      g.F1[i] = z4;
      g.type[i] = 0;
      if (g.v) g.v[i] = z4;
      if (g.vd) {
        const SysInt &S = g.sys[m.sys];
        const size_t n = S.natoms, dst = (size_t)S.vd0 + off;
        g.vd[dst] = 0.0;
        g.vd[dst + n] = 0.0;
        g.vd[dst + 2 * n] = 0.0;
      }
    }
    return;
  }
  for (uint32_t t = threadIdx.x; t < m.n; t += kIntThreads) {
    const uint32_t off = m.k * kIntAtoms + t;  // atom within its system
    const uint32_t i = m.i0 + t, o = q.o_atom0 + off;
    g.r[i] = g.o_r[o];
    g.F0[i] = (q.fb0 ? g.o_F1 : g.o_F0)[o];
    g.F1[i] = (q.fb1 ? g.o_F1 : g.o_F0)[o];
    g.minv[i] = g.o_minv[o];
    g.mass[i] = g.o_mass[o];
    g.type[i] = g.o_type[o];
    if (g.v) g.v[i] = g.o_v[o];
    if (g.vd) {
      // per-system planes x[n], y[n], z[n] starting at 3 x the system's first atom
      const SysInt &S = g.sys[m.sys];
      const size_t n = S.natoms, dst = (size_t)S.vd0 + off, src = 3 * (size_t)q.o_atom0 + off;
      g.vd[dst] = g.o_vd[src];
      g.vd[dst + n] = g.o_vd[src + n];
      g.vd[dst + 2 * n] = g.o_vd[src + 2 * n];
    }
  }
}

}  // namespace

cudaError_t launch_fill_sysid(const BlockMap *map, uint32_t nblocks, uint32_t *sysid,
                              cudaStream_t s) {
  if (!nblocks) return cudaSuccess;
  k_fill_sysid<<<nblocks, kIntThreads, 0, s>>>(map, sysid);
  return cudaGetLastError();
}

cudaError_t launch_gather_state(const GatherArgs &g, cudaStream_t s) {
  if (!g.nblocks) return cudaSuccess;
  k_gather_state<<<g.nblocks, kIntThreads, 0, s>>>(g);
  return cudaGetLastError();
}

uint32_t blocks_for(uint32_t natoms) { return (natoms + kIntAtoms - 1) / kIntAtoms; }

void make_block_map(const uint32_t *natoms, uint32_t nsys, BlockMap *map, uint32_t *blk0,
                    uint32_t *nblk) {
  uint32_t b = 0, atom0 = 0;
  for (uint32_t s = 0; s < nsys; ++s) {
    blk0[s] = b;
    nblk[s] = blocks_for(natoms[s]);
    for (uint32_t k = 0; k < nblk[s]; ++k) {
      const uint32_t i0 = atom0 + k * kIntAtoms;
      const uint32_t n = natoms[s] - k * kIntAtoms;
      map[b++] = BlockMap{s, i0, n < (uint32_t)kIntAtoms ? n : (uint32_t)kIntAtoms, k};
    }
    atom0 += natoms[s];
  }
}

#define PB_LAUNCH(kern, ...)                                                    \
  do {                                                                          \
    if (!a.nblocks) return cudaSuccess;                                         \
    kern<<<a.nblocks, kIntThreads, 0, s>>>(__VA_ARGS__);                        \
    return cudaGetLastError();                                                  \
  } while (0)

cudaError_t launch_vv(const IntegrateArgs &a, cudaStream_t s) {
  if (!a.nblocks) return cudaSuccess;
  return launch_pdl(k_vv, dim3(a.nblocks), dim3(kIntThreads), 0, s, a);
}
cudaError_t launch_wrap(const IntegrateArgs &a, cudaStream_t s) { PB_LAUNCH(k_wrap, a); }
cudaError_t launch_mv2(const IntegrateArgs &a, cudaStream_t s) { PB_LAUNCH(k_mv2, a); }
cudaError_t launch_fv(const IntegrateArgs &a, cudaStream_t s) { PB_LAUNCH(k_fv, a); }
cudaError_t launch_scale(const IntegrateArgs &a, const double *f, cudaStream_t s) {
  PB_LAUNCH(k_scale, a, f);
}

cudaError_t launch_gauss(const IntegrateArgs &a, cudaStream_t s) {
  if (!a.nblocks) return cudaSuccess;
  cudaError_t e = launch_pdl(k_gauss_a, dim3(a.nblocks), dim3(kIntThreads), 0, s, a);
  if (e == cudaSuccess) e = launch_pdl(k_gauss_b, dim3(a.nblocks), dim3(kIntThreads), 0, s, a);
  return e;
}

cudaError_t launch_adjust(const IntegrateArgs &a, const double *v1, cudaStream_t s) {
  if (!a.nblocks) return cudaSuccess;
  k_vstats<<<a.nblocks, kIntThreads, 0, s>>>(a);
  k_vapply<<<a.nblocks, kIntThreads, 0, s>>>(a, v1);
  return cudaGetLastError();
}

cudaError_t launch_euler(const IntegrateArgs &a, const float4 *F, float dt, cudaStream_t s) {
  PB_LAUNCH(k_euler, a, F, dt);
}

cudaError_t launch_sd_move(const IntegrateArgs &a, const float4 *F, float alpha, float max_disp,
                           cudaStream_t s) {
  PB_LAUNCH(k_sd_move, a, F, alpha, max_disp);
}

cudaError_t launch_correct_force(const IntegrateArgs &a, float4 *F, const double *lambda,
                                 cudaStream_t s) {
  PB_LAUNCH(k_correct, a, F, lambda);
}

cudaError_t launch_energy_total(const double *partials, const uint32_t *item0, uint32_t nsys,
                                DevScalars *sc, cudaStream_t s) {
  if (!nsys) return cudaSuccess;
  k_energy_total<<<nsys, kIntThreads, 0, s>>>(partials, item0, sc);
  return cudaGetLastError();
}

}  // namespace pb
