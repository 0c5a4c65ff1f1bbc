// Shared device-side types and helpers for the LJ cell-list step.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace pb {

constexpr int kMaxTypes = 8;
constexpr uint32_t kNone = 0xffffffffu;
// Neighbour cell or column outside an open box (the reference's UINT_MAX in
// its block-neighbour table).
constexpr uint32_t kNoCell = 0xffffffffu;

// Device status bits, OR-ed into a per-system status word.  No kernel traps;
// the host reads the word and turns it into a pb_status.
enum StatusBits : uint32_t {
  kStatusSmemOverflow = 1u << 0,   // a force CTA fell back to global loads
  kStatusNonFinite = 1u << 1,      // a NaN/Inf reached a reduction
  kStatusWaitTimeout = 1u << 2,    // a bounded wait gave up
  kStatusCellOverflow = 1u << 3,   // a cell held more atoms than a kernel supports
  kStatusNoConverge = 1u << 4,     // thermostat solve failed
  kStatusNlistOverflow = 1u << 5,  // a neighbour-list row outgrew its capacity
  kStatusStaleList = 1u << 6,      // an atom moved more than half the list skin since the build
};

// Cell grid of one periodic box, bit-compatible with cudaCutoffBlock:
// blocknum = floor(L / rmax) in FP32, blocklen = L / blocknum in FP32.
struct Grid {
  int n[3];          // cells per dimension (nx, ny, nz)
  float len[3];      // cell edge (blocklen)
  float lo[3];       // box minimum corner (cellmin)
  float L[3];        // box lengths (xmax - xmin etc., FP32)
  uint32_t ncells;
  int periodic;      // 0: open boundaries (no images, no wrap)
};

// Lennard-Jones parameters per ordered type pair, row-major [ti * nt + tj].
struct LJTable {
  int nt;
  float s2[kMaxTypes * kMaxTypes];    // sigma^2
  float e24[kMaxTypes * kMaxTypes];   // 24 epsilon
  float e4[kMaxTypes * kMaxTypes];    // 4 epsilon (energy)
  float rc2[kMaxTypes * kMaxTypes];   // cutoff^2 (the reference uses one rmax2)
  float ushift[kMaxTypes * kMaxTypes];  // U(rc), for the shifted energy
};

// ---- programmatic dependent launch -------------------------------------------
// The kernels of a step are launched with programmatic stream serialisation,
// so that a kernel's CTAs are scheduled while its predecessor drains.  Every
// such kernel calls pdl_enter() before anything else: it waits until the
// predecessor has finished and its memory is visible (the same ordering as a
// plain launch), then lets its own successor be scheduled.
#ifdef __CUDACC__
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Launch `k` with programmatic stream serialisation; the kernel must begin
// with pdl_enter().
template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                       Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k, args...);
}
#endif

// ---- small device helpers ---------------------------------------------------
#ifdef __CUDACC__

__device__ __forceinline__ float rcp_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// Cell index of one coordinate, exactly as calcBID_F4 (kernelfuncs.cu:807-841):
// IEEE single-precision (x - lo) / len, truncated with saturation, then the
// two clamps d == n -> n - 1 and d > n -> 0.
__device__ __forceinline__ int cell_coord(float x, float lo, float len, int n) {
  uint32_t d = __float2uint_rz(__fdiv_rn(__fsub_rn(x, lo), len));
  if (d == (uint32_t)n) {
    d = n - 1;
  } else if (d > (uint32_t)n) {
    d = 0;
  }
  return (int)d;
}

// Periodic wrap into [c0, c1) as applyPeriodicCondition_F4
// (kernelfuncs.cu:87-139), in the same FP32 operation order.
__device__ __forceinline__ float wrap_coord(float x, float c0, float c1, float L) {
  const float d0 = __fsub_rn(c0, x);
  if (d0 > 0.0f) {
    const int l0 = (int)__fdiv_rn(d0, L) + 1;
    x = __fadd_rn(x, __fmul_rn((float)l0, L));
  }
  const float d1 = __fsub_rn(x, c1);
  if (d1 >= 0.0f) {
    const int l1 = (int)__fdiv_rn(d1, L) + 1;
    x = __fsub_rn(x, __fmul_rn((float)l1, L));
  }
  return x;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum of NV doubles with a fixed reduction order; result valid in
// thread 0.  `scratch` needs NV * 32 doubles of shared memory.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double *scratch) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k) v[k] = warp_sum(v[k]);
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) scratch[k * 32 + warp] = v[k];
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double t = lane < nw ? scratch[k * 32 + lane] : 0.0;
      v[k] = warp_sum(t);
    }
  }
  __syncthreads();
}

// "Last block finishes the reduction": every block writes NV partial sums to
// partials[blockIdx.x * NV + k]; the block that arrives last sums all
// partials in block order (deterministic for a given grid) and returns true
// in thread 0 with the totals in `tot`.  `counter` must start at 0 and is
// reset by the last block.
template <int NV>
__device__ __forceinline__ bool last_block_total(const double (&mine)[NV], double *partials,
                                                 unsigned int *counter, double (&tot)[NV],
                                                 double *scratch) {
  __shared__ bool is_last;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) partials[(size_t)blockIdx.x * NV + k] = mine[k];
    __threadfence();
    const unsigned int ticket = atomicAdd(counter, 1u);
    is_last = (ticket == gridDim.x - 1);
  }
  __syncthreads();
  if (!is_last) return false;
  __threadfence();
  double acc[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k) acc[k] = 0.0;
  for (uint32_t b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
#pragma unroll
    for (int k = 0; k < NV; ++k) acc[k] += __ldcg(&partials[(size_t)b * NV + k]);
  }
  block_sum<NV>(acc, scratch);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) tot[k] = acc[k];
    *counter = 0;
  }
  return threadIdx.x == 0;
}
#endif  // __CUDACC__

}  // namespace pb
