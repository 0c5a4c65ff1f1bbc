// Cell-list build: bin every atom into its cell, counting-sort the atoms by
// packed cell key, and gather sorted positions.
//
// Replaces cudaCutoffBlock::calcBlockID + cudaSortedPositions::calcBlockID
// (cudaCutoffBlock.cu:233-258, cudaSortedPositions.cu:27-30), i.e. calcBID_F4,
// sortByBID_M1, the single-CTA sortByBID, makeBindex and copyWithIndex
// (kernelfuncs.cu:807-932).  The cell of each atom is computed with the same
// FP32 arithmetic as calcBID_F4, so cell membership is bit-identical; the
// within-cell order is canonical -- ascending z, ties by particle id -- instead
// of the reference's history-dependent order.  Because the cell index is a
// monotone function of z, every (x, y) column of cells is then sorted by z,
// which the force kernel uses to cut z windows by binary search.
//
// Kernels, in launch order:
//   k_bin       read r (16 B/atom), write key + within-cell ticket (8 B/atom)
//   k_scan_*    exclusive scan of per-cell counts -> start[], zero the counts
//   k_scatter   pid_tmp[start[key] + ticket] = i
//   k_canon     one warp per two cells: order members by (z, particle id), write
//               pid, slot, the sorted position float4 (type id in .w) and its
//               structure-of-arrays mirror (x, y, z, type) for the force kernel
#include "md.cuh"

namespace pb {
namespace {

constexpr int kScanTile = 4096;  // counts per scan tile (1024 threads x 4)

__device__ __forceinline__ uint32_t system_of(const CellBufs &b, uint32_t i) {
  return b.sysid ? b.sysid[i] : 0u;
}

__global__ void __launch_bounds__(256) k_bin(CellBufs b) {
  pdl_enter();
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= b.N) return;
  const SysDesc &S = b.sys[system_of(b, i)];
  const float4 p = b.r[i];
  const int d0 = cell_coord(p.x, S.g.lo[0], S.g.len[0], S.g.n[0]);
  const int d1 = cell_coord(p.y, S.g.lo[1], S.g.len[1], S.g.n[1]);
  const int d2 = cell_coord(p.z, S.g.lo[2], S.g.len[2], S.g.n[2]);
  const uint32_t rank = b.colrank[S.col0 + d0 * S.g.n[1] + d1];
  const uint32_t key = S.cell0 + rank * (uint32_t)S.g.n[2] + (uint32_t)d2;
  b.key[i] = key;
  b.within[i] = atomicAdd(&b.count[key], 1u);
}

// Tile-local exclusive scan of kScanTile counts; writes the tile total and
// zeroes the counts for the next build.
__global__ void __launch_bounds__(1024) k_scan_tiles(CellBufs b) {
  pdl_enter();
  __shared__ uint32_t warp_tot[32];
  const uint32_t base = blockIdx.x * kScanTile + threadIdx.x * 4;
  uint32_t c[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const uint32_t idx = base + k;
    c[k] = idx < b.ncells ? b.count[idx] : 0u;
  }
  uint32_t sum = c[0] + c[1] + c[2] + c[3];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t incl = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) warp_tot[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = warp_tot[lane];
    uint32_t wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += t;
    }
    warp_tot[lane] = wi - w;  // exclusive prefix of warp totals
    if (lane == 31) b.tilesum[blockIdx.x] = wi;
  }
  __syncthreads();
  uint32_t run = warp_tot[warp] + incl - sum;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const uint32_t idx = base + k;
    if (idx < b.ncells) {
      b.start[idx] = run;
      b.count[idx] = 0u;
    }
    run += c[k];
  }
}

// Exclusive scan of the tile totals (single block; up to 1024 * 32 tiles).
__global__ void __launch_bounds__(1024) k_scan_top(CellBufs b, uint32_t ntiles) {
  pdl_enter();
  __shared__ uint32_t warp_tot[32];
  __shared__ uint32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (uint32_t base = 0; base < ntiles; base += blockDim.x) {
    const uint32_t idx = base + threadIdx.x;
    const uint32_t v = idx < ntiles ? b.tilesum[idx] : 0u;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      const uint32_t w = warp_tot[lane];
      uint32_t wi = w;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, wi, o);
        if (lane >= o) wi += t;
      }
      warp_tot[lane] = wi - w;
    }
    __syncthreads();
    const uint32_t excl = carry + warp_tot[warp] + incl - v;
    if (idx < ntiles) b.tilesum[idx] = excl;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = excl + v;
    __syncthreads();
  }
  if (threadIdx.x == 0) b.start[b.ncells] = carry;
}

__global__ void __launch_bounds__(256) k_scan_add(CellBufs b) {
  pdl_enter();
  const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx < b.ncells) b.start[idx] += b.tilesum[idx / kScanTile];
}

__global__ void __launch_bounds__(256) k_scatter(CellBufs b) {
  pdl_enter();
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= b.N) return;
  b.pid_tmp[b.start[b.key[i]] + b.within[i]] = i;
}

// SoA mirror of sorted slot s (atom `me`, cell `key`): the system's sorted
// atom s - atom0 goes to mirror0 + (s - atom0).  An atom with a NaN or
// infinite coordinate (a simulation that has blown up) is mirrored far away
// in x and y, at the top edge of its cell in z, so that the force kernel never
// finds it within range while every column stays sorted in z.
__device__ __forceinline__ void write_mirror(const CellBufs &b, uint32_t me, uint32_t s,
                                             const float4 &p, uint32_t key) {
  const SysDesc &S = b.sys[system_of(b, me)];
  const uint32_t m = S.mirror0 + (s - S.atom0);
  float x = p.x, y = p.y, z = p.z;
  if (!isfinite(x) || !isfinite(y) || !isfinite(z)) {
    const uint32_t d2 = (key - S.cell0) % (uint32_t)S.g.n[2];
    x = 1e30f;
    y = 1e30f;
    z = S.g.lo[2] + (float)(d2 + 1) * S.g.len[2];
  }
  b.xs[m] = x;
  b.ys[m] = y;
  b.zs[m] = z;
  b.ts[m] = (uint32_t)b.type[me];
}

// Order key of a z coordinate: monotone in z for all non-NaN values (-0 and
// +0 share a key, as they compare equal), every NaN after +Inf.  Ranking by
// (key, particle id) is a strict total order, so the ranks of a cell's members
// are a permutation of 0 .. n - 1 even when a coordinate is NaN: no slot is
// left unwritten and none is written twice.
__device__ __forceinline__ uint32_t z_key(float z) {
  if (z != z) return 0xffffffffu;
  uint32_t u = __float_as_uint(z);
  if (u == 0x80000000u) u = 0u;
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__device__ __forceinline__ bool canon_before(uint32_t ka, uint32_t a, uint32_t kb, uint32_t b) {
  return ka < kb || (ka == kb && a < b);
}

// Rank of every member of one cell by (z, particle id), one lane per member,
// among the `width` lanes starting at lane `base` (width 16 or 32).  The rank
// of a member is the number of members before it in that order, which orders
// each cell canonically without depending on the atomic tickets of k_bin.
__device__ __forceinline__ void canon_cell(const CellBufs &b, uint32_t s0, uint32_t n, int li,
                                           int base, uint32_t lanes_n, uint32_t key) {
  const uint32_t me = li < (int)n ? b.pid_tmp[s0 + li] : kNone;
  const float4 p = li < (int)n ? b.r[me] : make_float4(0.f, 0.f, 0.f, 0.f);
  const uint32_t kz = z_key(p.z);
  uint32_t rank = 0;
  for (uint32_t k = 0; k < lanes_n; ++k) {
    const uint32_t other = __shfl_sync(0xffffffffu, me, base + (int)k);
    const uint32_t ko = __shfl_sync(0xffffffffu, kz, base + (int)k);
    rank += (k < n && canon_before(ko, other, kz, me)) ? 1u : 0u;
  }
  if (li < (int)n) {
    const uint32_t s = s0 + rank;
    b.pid[s] = me;
    b.slot[me] = s;
    b.rs[s] = make_float4(p.x, p.y, p.z, __int_as_float((int)b.type[me]));
    if (b.xs) write_mirror(b, me, s, p, key);
  }
}

// Cells with more than 32 members: O(n^2 / 32) ranking straight from global memory.
__device__ void canon_large(const CellBufs &b, uint32_t s0, uint32_t n, int lane, uint32_t key) {
  for (uint32_t a = lane; a < n; a += 32) {
    const uint32_t me = b.pid_tmp[s0 + a];
    const float4 p = b.r[me];
    const uint32_t kz = z_key(p.z);
    uint32_t rank = 0;
    for (uint32_t k = 0; k < n; ++k) {
      const uint32_t other = b.pid_tmp[s0 + k];
      rank += canon_before(z_key(b.r[other].z), other, kz, me) ? 1u : 0u;
    }
    const uint32_t s = s0 + rank;
    b.pid[s] = me;
    b.slot[me] = s;
    b.rs[s] = make_float4(p.x, p.y, p.z, __int_as_float((int)b.type[me]));
    if (b.xs) write_mirror(b, me, s, p, key);
  }
}

// One warp per pair of packed cells: when both hold at most 16 members, each
// half-warp orders one of them; otherwise the whole warp orders one, then the
// other.
__global__ void __launch_bounds__(256) k_canon(CellBufs b) {
  pdl_enter();
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const uint32_t c0 = 2 * warp;
  if (c0 >= b.ncells) return;
  const bool two = c0 + 1 < b.ncells;
  const uint32_t s0 = b.start[c0], s1 = b.start[c0 + 1];
  const uint32_t s2 = two ? b.start[c0 + 2] : s1;
  const uint32_t n0 = s1 - s0, n1 = s2 - s1;
  if (n0 <= 16 && n1 <= 16) {
    const int half = lane >> 4;
    canon_cell(b, half ? s1 : s0, half ? n1 : n0, lane & 15, half * 16, max(n0, n1),
               c0 + (uint32_t)half);
    return;
  }
  for (int k = 0; k < (two ? 2 : 1); ++k) {
    const uint32_t sb = k ? s1 : s0, n = k ? n1 : n0;
    if (n <= 32)
      canon_cell(b, sb, n, lane, 0, n, c0 + (uint32_t)k);
    else
      canon_large(b, sb, n, lane, c0 + (uint32_t)k);
  }
}

}  // namespace

cudaError_t launch_cell_build(const CellBufs &b, cudaStream_t s) {
  if (b.N == 0) return cudaSuccess;
  const uint32_t nb = (b.N + 255) / 256;
  cudaError_t e = launch_pdl(k_bin, dim3(nb), dim3(256), 0, s, b);
  const uint32_t ntiles = (b.ncells + kScanTile - 1) / kScanTile;
  if (e == cudaSuccess) e = launch_pdl(k_scan_tiles, dim3(ntiles), dim3(1024), 0, s, b);
  if (e == cudaSuccess) e = launch_pdl(k_scan_top, dim3(1), dim3(1024), 0, s, b, ntiles);
  if (e == cudaSuccess)
    e = launch_pdl(k_scan_add, dim3((b.ncells + 255) / 256), dim3(256), 0, s, b);
  if (e == cudaSuccess) e = launch_pdl(k_scatter, dim3(nb), dim3(256), 0, s, b);
  const uint64_t canon_threads = (uint64_t)((b.ncells + 1) / 2) * 32;
  if (e == cudaSuccess)
    e = launch_pdl(k_canon, dim3((uint32_t)((canon_threads + 255) / 256)), dim3(256), 0, s, b);
  return e;
}

}  // namespace pb
