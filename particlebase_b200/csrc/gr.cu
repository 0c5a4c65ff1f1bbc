// Radial distribution function: pair counts per distance bin.
//
// Replaces cudaCalcGR::calcgr (cudaCalcGR.cu:85-116) with the pair kernel
// calcF_IJpairWithBlock5_F4<calcGR_F4> (kerneltemplate.hh:423-512,
// kernelinline.hh:433-449): every unordered pair of atoms, minimum image,
// bin j = trunc(r / rstep + 1/2), counted when 0 < j < rnum.  The reference
// walks every pair of cell blocks (makePairInfo, cudaCalcGR.cu:43-83), so the
// work is all pairs whatever rmax is; here the pairs are tiles of 128 x 128
// atoms (tile I against tiles J >= I, j > i inside a diagonal tile), counted in
// a per-CTA shared-memory histogram and added to the global counts with
// 64-bit integer atomics, so the result does not depend on scheduling.
//
// Arithmetic: FP32 round-to-nearest with no fused multiply-add (explicit
// __fmul_rn / __fadd_rn / __fsqrt_rn), r^2 = (dx^2 + dy^2) + dz^2, and the
// exact minimum image (the coordinate above the box middle moved down by L
// first).  The oracle restates exactly these operations.
#include "md.cuh"

namespace pb {
namespace {

constexpr int kGrTile = 128;

__device__ __forceinline__ float image_delta(float xi, float xj, float L, float hL) {
  const float d = __fsub_rn(xi, xj);
  if (d > hL) return __fsub_rn(__fsub_rn(xi, L), xj);
  if (d < -hL) return __fsub_rn(xi, __fsub_rn(xj, L));
  return d;
}

__global__ void __launch_bounds__(kGrTile) k_gr(const float4 *__restrict__ r, uint32_t N,
                                                float Lx, float Ly, float Lz, float inv,
                                                uint32_t rnum, unsigned long long *counts) {
  extern __shared__ uint32_t hist[];  // rnum bins
  __shared__ float4 tj[kGrTile];
  const uint32_t I = blockIdx.y, J = blockIdx.x;
  if (J < I) return;  // each unordered tile pair once
  for (uint32_t b = threadIdx.x; b < rnum; b += blockDim.x) hist[b] = 0u;
  const uint32_t j0 = J * kGrTile;
  {
    const uint32_t j = j0 + threadIdx.x;
    tj[threadIdx.x] = j < N ? r[j] : make_float4(0.f, 0.f, 0.f, 0.f);
  }
  __syncthreads();
  const uint32_t i = I * kGrTile + threadIdx.x;
  if (i < N) {
    const float4 p = r[i];
    const float hx = 0.5f * Lx, hy = 0.5f * Ly, hz = 0.5f * Lz;
    const uint32_t jn = min((uint32_t)kGrTile, N - j0);
    for (uint32_t k = I == J ? threadIdx.x + 1 : 0; k < jn; ++k) {
      const float4 q = tj[k];
      const float dx = image_delta(p.x, q.x, Lx, hx);
      const float dy = image_delta(p.y, q.y, Ly, hy);
      const float dz = image_delta(p.z, q.z, Lz, hz);
      const float r2 =
          __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
      const float x = __fadd_rn(__fmul_rn(__fsqrt_rn(r2), inv), 0.5f);
      if (x < (float)rnum) {  // also keeps the conversion in range
        const uint32_t b = (uint32_t)x;
        if (b > 0u && b < rnum) atomicAdd(&hist[b], 1u);
      }
    }
  }
  __syncthreads();
  for (uint32_t b = threadIdx.x; b < rnum; b += blockDim.x)
    if (hist[b]) atomicAdd(&counts[b], (unsigned long long)hist[b]);
}

}  // namespace

uint32_t gr_max_bins() { return 16384; }

cudaError_t launch_gr(const float4 *r, uint32_t N, const float L[3], float inv, uint32_t rnum,
                      unsigned long long *counts, cudaStream_t s) {
  if (N == 0 || rnum == 0) return cudaSuccess;
  const uint32_t T = (N + kGrTile - 1) / kGrTile;
  const size_t smem = sizeof(uint32_t) * rnum;
  cudaError_t e = cudaFuncSetAttribute(k_gr, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  k_gr<<<dim3(T, T), kGrTile, smem, s>>>(r, N, L[0], L[1], L[2], inv, rnum, counts);
  return cudaGetLastError();
}

}  // namespace pb
