// Velocity Verlet, Gaussian isokinetic thermostat, periodic wrap and the
// FP64 reductions around them, for one system in particle order.
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

constexpr int kThreads = 256;

__device__ __forceinline__ float4 load_v(const IntegrateArgs &a, uint32_t i) {
  if (a.vd) return make_float4((float)a.vd[i], (float)a.vd[i + a.N], (float)a.vd[i + 2 * a.N], 0.f);
  return a.v[i];
}

__device__ __forceinline__ void wrap3(const IntegrateArgs &a, float4 &p) {
  p.x = wrap_coord(p.x, a.c0[0], a.c1[0], a.L[0]);
  p.y = wrap_coord(p.y, a.c0[1], a.c1[1], a.L[1]);
  p.z = wrap_coord(p.z, a.c0[2], a.c1[2], a.L[2]);
}

__global__ void __launch_bounds__(kThreads) k_vv(IntegrateArgs a) {
  __shared__ double red[32];
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  double mv2 = 0;
  if (i < a.N) {
    const float dt2 = a.dt * 0.5f;
    const float h = dt2 * a.minv[i];  // dt / 2m
    const float4 F = a.F[i], Fo = a.Fold[i];
    float4 v = a.v[i];
    v.x += (F.x + Fo.x) * h;
    v.y += (F.y + Fo.y) * h;
    v.z += (F.z + Fo.z) * h;
    v.w = 0.f;
    const float h2 = h * a.dt;
    float4 p = a.r[i];
    p.x += v.x * a.dt + F.x * h2;
    p.y += v.y * a.dt + F.y * h2;
    p.z += v.z * a.dt + F.z * h2;
    if (a.wrap) wrap3(a, p);
    a.v[i] = v;
    a.r[i] = p;
    mv2 = (double)a.mass[i] *
          ((double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z);
  }
  double m[1] = {mv2}, tot[1];
  block_sum<1>(m, red);
  if (last_block_total<1>(m, a.partials, &a.sc->counter[0], tot, red)) {
    a.sc->mv2 = tot[0];
    if (!isfinite(tot[0])) atomicOr(a.status, kStatusNonFinite);
  }
}

// A for atom i (FP64), identical arithmetic in both Gaussian passes.
__device__ __forceinline__ void gauss_A(const IntegrateArgs &a, uint32_t i, double xi_old,
                                        double A[3], float4 &F) {
  const float h = (a.dt * 0.5f) * a.minv[i];
  F = a.F[i];
  const float4 Fo = a.Fold[i];
  double v0[3];
  if (a.vd) {
    v0[0] = a.vd[i];
    v0[1] = a.vd[i + a.N];
    v0[2] = a.vd[i + 2 * a.N];
  } else {
    const float4 v = a.v[i];
    v0[0] = v.x;
    v0[1] = v.y;
    v0[2] = v.z;
  }
  const double hx = (double)a.dt * 0.5 * xi_old;
  A[0] = v0[0] + (double)(F.x + Fo.x) * h - v0[0] * hx;
  A[1] = v0[1] + (double)(F.y + Fo.y) * h - v0[1] * hx;
  A[2] = v0[2] + (double)(F.z + Fo.z) * h - v0[2] * hx;
}

__global__ void __launch_bounds__(kThreads) k_gauss_a(IntegrateArgs a) {
  __shared__ double red[2 * 32];
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const double xi_old = a.sc->xi_old;
  double s[2] = {0, 0};
  if (i < a.N) {
    double A[3];
    float4 F;
    gauss_A(a, i, xi_old, A, F);
    s[0] = (double)F.x * A[0] + (double)F.y * A[1] + (double)F.z * A[2];
    s[1] = (double)a.mass[i] * (A[0] * A[0] + A[1] * A[1] + A[2] * A[2]);
  }
  double tot[2];
  block_sum<2>(s, red);
  if (last_block_total<2>(s, a.partials, &a.sc->counter[1], tot, red)) {
    const double hdt = 0.5 * (double)a.dt;
    const double c = tot[1] > 0 ? tot[0] / tot[1] : 0.0;
    double xi = (xi_old == 0.0) ? c : c / (1.0 - c * hdt);
    if (!isfinite(xi) || !isfinite(tot[0]) || !isfinite(tot[1])) {
      atomicOr(a.status, kStatusNonFinite | kStatusNoConverge);
      xi = 0.0;
    }
    a.sc->sum_fa = tot[0];
    a.sc->sum_ma2 = tot[1];
    a.sc->xi_new = xi;
  }
}

__global__ void __launch_bounds__(kThreads) k_gauss_b(IntegrateArgs a) {
  __shared__ double red[32];
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const double xi_old = a.sc->xi_old;
  const double xi = a.sc->xi_new;
  double mv2 = 0;
  if (i < a.N) {
    double A[3];
    float4 F;
    gauss_A(a, i, xi_old, A, F);
    const double dt = a.dt;
    const double inv = (xi_old == 0.0) ? 1.0 : 1.0 / (1.0 + xi * 0.5 * dt);
    const double v[3] = {A[0] * inv, A[1] * inv, A[2] * inv};
    const double cv = dt - xi * 0.5 * dt * dt;
    const double cf = 0.5 * dt * dt * (double)a.minv[i];
    float4 p = a.r[i];
    p.x = (float)((double)p.x + v[0] * cv + (double)F.x * cf);
    p.y = (float)((double)p.y + v[1] * cv + (double)F.y * cf);
    p.z = (float)((double)p.z + v[2] * cv + (double)F.z * cf);
    if (a.wrap) wrap3(a, p);
    a.r[i] = p;
    if (a.vd) {
      a.vd[i] = v[0];
      a.vd[i + a.N] = v[1];
      a.vd[i + 2 * a.N] = v[2];
      mv2 = (double)a.mass[i] * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    } else {
      const float4 vf = make_float4((float)v[0], (float)v[1], (float)v[2], 0.f);
      a.v[i] = vf;
      mv2 = (double)a.mass[i] * ((double)vf.x * vf.x + (double)vf.y * vf.y + (double)vf.z * vf.z);
    }
  }
  double m[1] = {mv2}, tot[1];
  block_sum<1>(m, red);
  if (last_block_total<1>(m, a.partials, &a.sc->counter[2], tot, red)) {
    a.sc->mv2 = tot[0];
    a.sc->xi_old = xi;  // every other block has finished reading xi_old
    if (!isfinite(tot[0])) atomicOr(a.status, kStatusNonFinite);
  }
}

__global__ void __launch_bounds__(kThreads) k_wrap(IntegrateArgs a) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.N) return;
  float4 p = a.r[i];
  wrap3(a, p);
  a.r[i] = p;
}

__global__ void __launch_bounds__(kThreads) k_mv2(IntegrateArgs a) {
  __shared__ double red[32];
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  double m[1] = {0};
  if (i < a.N) {
    const float4 v = load_v(a, i);
    double vx = v.x, vy = v.y, vz = v.z;
    if (a.vd) {
      vx = a.vd[i];
      vy = a.vd[i + a.N];
      vz = a.vd[i + 2 * a.N];
    }
    m[0] = (double)a.mass[i] * (vx * vx + vy * vy + vz * vz);
  }
  double tot[1];
  block_sum<1>(m, red);
  if (last_block_total<1>(m, a.partials, &a.sc->counter[0], tot, red)) a.sc->mv2 = tot[0];
}

__global__ void __launch_bounds__(kThreads) k_fv(IntegrateArgs a) {
  __shared__ double red[32];
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  double m[1] = {0};
  if (i < a.N) {
    const float4 F = a.F[i];
    double vx, vy, vz;
    if (a.vd) {
      vx = a.vd[i];
      vy = a.vd[i + a.N];
      vz = a.vd[i + 2 * a.N];
    } else {
      const float4 v = a.v[i];
      vx = v.x;
      vy = v.y;
      vz = v.z;
    }
    m[0] = (double)F.x * vx + (double)F.y * vy + (double)F.z * vz;
  }
  double tot[1];
  block_sum<1>(m, red);
  if (last_block_total<1>(m, a.partials, &a.sc->counter[3], tot, red)) a.sc->fv = tot[0];
}

__global__ void __launch_bounds__(kThreads) k_scale(IntegrateArgs a, double s) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.N) return;
  if (a.vd) {
    a.vd[i] *= s;
    a.vd[i + a.N] *= s;
    a.vd[i + 2 * a.N] *= s;
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

// adjustVelocity_F4 / adjustVelocity_VD (kernelfuncs.cu:546-699): per axis,
// subtract the mean and scale to standard deviation v1.  Pass 1: sums.
__global__ void __launch_bounds__(kThreads) k_vstats(IntegrateArgs a) {
  __shared__ double red[6 * 32];
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  double s[6] = {0, 0, 0, 0, 0, 0};
  if (i < a.N) {
    double w[3];
    if (a.vd) {
      w[0] = a.vd[i];
      w[1] = a.vd[i + a.N];
      w[2] = a.vd[i + 2 * a.N];
    } else {
      const float4 v = a.v[i];
      w[0] = v.x;
      w[1] = v.y;
      w[2] = v.z;
    }
    for (int k = 0; k < 3; ++k) {
      s[k] = w[k];
      s[3 + k] = w[k] * w[k];
    }
  }
  double tot[6];
  block_sum<6>(s, red);
  if (last_block_total<6>(s, a.partials, &a.sc->counter[3], tot, red)) {
    for (int k = 0; k < 6; ++k) a.sc->vstat[k] = tot[k];
  }
}

__global__ void __launch_bounds__(kThreads) k_vapply(IntegrateArgs a, double v1) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.N) return;
  const double n = (double)a.N;
  double mean[3], sc[3];
  for (int k = 0; k < 3; ++k) {
    mean[k] = a.sc->vstat[k] / n;
    const double var = a.sc->vstat[3 + k] / n - mean[k] * mean[k];
    sc[k] = var > 0 ? v1 / sqrt(var) : 0.0;
  }
  if (a.vd) {
    for (int k = 0; k < 3; ++k) a.vd[i + k * a.N] = (a.vd[i + k * a.N] - mean[k]) * sc[k];
  } else {
    float4 v = a.v[i];
    v.x = (float)((v.x - mean[0]) * sc[0]);
    v.y = (float)((v.y - mean[1]) * sc[1]);
    v.z = (float)((v.z - mean[2]) * sc[2]);
    a.v[i] = v;
  }
}

__global__ void __launch_bounds__(kThreads) k_energy_total(const double *partials, uint32_t n,
                                                          DevScalars *sc) {
  __shared__ double red[4 * 32];
  double s[4] = {0, 0, 0, 0};
  for (uint32_t b = threadIdx.x; b < n; b += blockDim.x) {
    s[0] += partials[(size_t)b * 4 + 0];
    s[1] += partials[(size_t)b * 4 + 1];
    s[2] += partials[(size_t)b * 4 + 2];
    s[3] += partials[(size_t)b * 4 + 3];
  }
  block_sum<4>(s, red);
  if (threadIdx.x == 0) {
    sc->pe = s[0];
    sc->pe_shift = s[1];
    sc->virial = s[2];
    sc->npairs = s[3];
  }
}

}  // namespace

uint32_t integrate_blocks(uint32_t N) { return (N + kThreads - 1) / kThreads; }

cudaError_t launch_vv(const IntegrateArgs &a, cudaStream_t s) {
  if (!a.N) return cudaSuccess;
  k_vv<<<integrate_blocks(a.N), kThreads, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_gauss(const IntegrateArgs &a, cudaStream_t s) {
  if (!a.N) return cudaSuccess;
  k_gauss_a<<<integrate_blocks(a.N), kThreads, 0, s>>>(a);
  k_gauss_b<<<integrate_blocks(a.N), kThreads, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_wrap(const IntegrateArgs &a, cudaStream_t s) {
  if (!a.N) return cudaSuccess;
  k_wrap<<<integrate_blocks(a.N), kThreads, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_mv2(const IntegrateArgs &a, cudaStream_t s) {
  if (!a.N) return cudaSuccess;
  k_mv2<<<integrate_blocks(a.N), kThreads, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_fv(const IntegrateArgs &a, cudaStream_t s) {
  if (!a.N) return cudaSuccess;
  k_fv<<<integrate_blocks(a.N), kThreads, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_scale(const IntegrateArgs &a, double factor, cudaStream_t s) {
  if (!a.N) return cudaSuccess;
  k_scale<<<integrate_blocks(a.N), kThreads, 0, s>>>(a, factor);
  return cudaGetLastError();
}

cudaError_t launch_adjust(const IntegrateArgs &a, double v1, cudaStream_t s) {
  if (!a.N) return cudaSuccess;
  k_vstats<<<integrate_blocks(a.N), kThreads, 0, s>>>(a);
  k_vapply<<<integrate_blocks(a.N), kThreads, 0, s>>>(a, v1);
  return cudaGetLastError();
}

cudaError_t launch_energy_total(const double *partials, uint32_t nparts, DevScalars *sc,
                                cudaStream_t s) {
  k_energy_total<<<1, kThreads, 0, s>>>(partials, nparts, sc);
  return cudaGetLastError();
}

}  // namespace pb
