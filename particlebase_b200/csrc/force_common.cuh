// Pieces shared by the two force kernels (force.cu, the full-shell kernel;
// force_half.cu, the half-shell kernel): work-item constants, the per-item LJ
// table, shared-memory access helpers, the bounded hand-off waits and the
// z-window searches.  Everything here has internal linkage in each file that
// includes it.
#pragma once

#include <cstdint>

#include "md.cuh"
#include "tma.cuh"

namespace pb {
namespace {

constexpr int kMaxSeg = 32;     // longest z run of one work item (cells)
constexpr int kListLen = 40;    // per-lane pair list entries
constexpr int kCopyBatch = 4;   // stage quads a producer thread loads before storing
constexpr int kChunk = 16;      // candidates a lane tests between list checks
constexpr int kWinCap = 48;     // clusters (or global-path tasks) per item
constexpr float kFar = 1e30f;   // pad-slot coordinate: never within range
constexpr float kNoAtom = -1e30f;  // coordinate of a padded home lane

static_assert(kListLen >= kChunk, "a chunk must fit an empty list");
static_assert(kChunk == 16, "the quad table layout holds chunks of 16 quads");

template <int NT>
struct LJLocal {
  float s2[NT * NT], e24[NT * NT], e4[NT * NT], rc2[NT * NT], ush[NT * NT];
  float sc_rc, sc_f0;  // soft-core mode: range and strength
};

// Pair force laws of the kernel.
constexpr int kModeLJ = 0;        // truncated LJ (the MD step)
constexpr int kModeCapped = 1;    // LJ with r^2 floored at (sigma/2)^2 (steepest descent)
constexpr int kModeSoftCore = 2;  // f0 cos(pi r / 2 rc) along r (initialAnnealing)

// One stage buffer: X, Y, Z planes and, with more than one type, a type plane.
struct Planes {
  float *X, *Y, *Z;
  uint32_t *T;
};

// Shared-memory access by 32-bit shared address.
__device__ __forceinline__ float4 lds_f4(uint32_t a) {
  float4 v;
  // not volatile: the stage is read-only while a cluster is computed, so the
  // compiler may schedule these loads freely
  asm("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
      : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
      : "r"(a));
  return v;
}

// Read-only global loads of 16 bytes (the sorted-position mirrors, which no
// kernel writes while the force kernel runs).
__device__ __forceinline__ float4 ldg_f4(const float *p) {
  float4 v;
  asm("ld.global.nc.v4.f32 {%0, %1, %2, %3}, [%4];"
      : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
      : "l"(p));
  return v;
}

__device__ __forceinline__ uint4 ldg_u4(const uint32_t *p) {
  uint4 v;
  asm("ld.global.nc.v4.u32 {%0, %1, %2, %3}, [%4];"
      : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
      : "l"(p));
  return v;
}

// Stage stores of the producers (ordered before their barrier, which is
// volatile too).
__device__ __forceinline__ void sts_f4(uint32_t a, float4 v) {
  asm volatile("st.shared.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(a), "f"(v.x), "f"(v.y), "f"(v.z),
               "f"(v.w));
}

__device__ __forceinline__ float lds_f32(uint32_t a) {
  float v;
  asm("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(a));
  return v;
}

// List entries are read after the warp's own stores (ordered by __syncwarp
// and the memory clobber of those stores), so this load is volatile.
__device__ __forceinline__ uint32_t lds_u16(uint32_t a) {
  unsigned short v;
  asm volatile("ld.shared.u16 %0, [%1];" : "=h"(v) : "r"(a) : "memory");
  return v;
}

__device__ __forceinline__ void sts_u16(uint32_t a, uint32_t v) {
  asm volatile("st.shared.u16 [%0], %1;" ::"r"(a), "h"((unsigned short)v) : "memory");
}

__device__ __forceinline__ uint32_t lds_u32(uint32_t a) {
  uint32_t v;
  asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"(a) : "memory");
  return v;
}

__device__ __forceinline__ void sts_u32(uint32_t a, uint32_t v) {
  asm volatile("st.shared.u32 [%0], %1;" ::"r"(a), "r"(v) : "memory");
}

// Position of flat quad u in a warp's quad table: within each chunk of 16,
// the 4 quads lane q tests (u = q, q + 4, q + 8, q + 12) are adjacent, so a
// lane fetches a chunk's quads with one 8-byte load.
__device__ __forceinline__ uint32_t table_pos(uint32_t u) {
  return (u & ~15u) | ((u & 3u) << 2) | ((u >> 2) & 3u);
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ const int kNeverAbort = 0;

// Bounded wait of the hand-off barriers: the polling thread sleeps between
// polls (up to 1 us each, at most `limit` polls, 2^22 by default), so waiting
// warps leave the issue slots to the warps that compute.  Gives up early when
// the CTA has aborted.
constexpr uint32_t kWaitPolls = 1u << 22;

__device__ __forceinline__ bool mbar_wait_or_abort(uint64_t *bar, uint32_t parity,
                                                   const volatile int *abort_flag,
                                                   uint32_t limit = kWaitPolls) {
  for (uint32_t it = 0; it < limit; ++it) {
    if (mbar_try_wait_sleep(bar, parity, 1000u)) return true;
    if (*abort_flag) return false;
  }
  return false;
}

__device__ __forceinline__ uint32_t lower_bound_z(const float *Z, uint32_t lo, uint32_t hi,
                                                  float key) {
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (Z[mid] < key) lo = mid + 1; else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ uint32_t upper_bound_z(const float *Z, uint32_t lo, uint32_t hi,
                                                  float key) {
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (Z[mid] <= key) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// Barrier of the kProd producer warps only (named barrier 1).
template <int kProd>
__device__ __forceinline__ void producer_sync() {
  asm volatile("bar.sync 1, %0;" ::"r"(kProd * 32) : "memory");
}

}  // namespace
}  // namespace pb
