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
// Two-kernel build (the engines):
//   k_bin_buckets  read r (16 B/atom); write key and the atom's id into its
//                  cell's bucket (members past the bucket's capacity go to an
//                  overflow list); count atoms per cell and per 64-cell tile
//                  with one atomic per distinct cell (tile) of a warp
//   k_canon_tiles  one block per 64-cell tile: the tile's first slot from the
//                  tile counts before it (no inter-block wait) and the starts
//                  of its cells; then its members ordered by (z, particle id),
//                  staged in shared memory, and pid, slot, the sorted position
//                  float4 (type id in .w) and its structure-of-arrays mirror
//                  (x, y, z, type) for the force kernel written
// Six-kernel build (the allocation-free entry point, which has no buckets):
//   k_bin       read r (16 B/atom), write key + within-cell ticket (8 B/atom)
//   k_scan_*    exclusive scan of per-cell counts -> start[], zero the counts
//   k_scatter   pid_tmp[start[key] + ticket] = i
//   k_canon     k_canon_tiles' ordering, one warp per two cells, members from
//               pid_tmp
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
__device__ __forceinline__ void write_mirror_of(const CellBufs &b, const SysDesc &S, uint32_t s,
                                                const float4 &p, uint32_t key, uint32_t type) {
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
  b.ts[m] = type;
}

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
__device__ __forceinline__ void canon_cell(const CellBufs &b, const uint32_t *mem, uint32_t s0,
                                           uint32_t n, int li, int base, uint32_t lanes_n,
                                           uint32_t key) {
  const uint32_t me = li < (int)n ? mem[li] : kNone;
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
__device__ void canon_large(const CellBufs &b, const uint32_t *mem, uint32_t s0, uint32_t n,
                            int lane, uint32_t key) {
  for (uint32_t a = lane; a < n; a += 32) {
    const uint32_t me = mem[a];
    const float4 p = b.r[me];
    const uint32_t kz = z_key(p.z);
    uint32_t rank = 0;
    for (uint32_t k = 0; k < n; ++k) {
      const uint32_t other = mem[k];
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
    const uint32_t sb = half ? s1 : s0;
    canon_cell(b, b.pid_tmp + sb, sb, half ? n1 : n0, lane & 15, half * 16, max(n0, n1),
               c0 + (uint32_t)half);
    return;
  }
  for (int k = 0; k < (two ? 2 : 1); ++k) {
    const uint32_t sb = k ? s1 : s0, n = k ? n1 : n0;
    if (n <= 32)
      canon_cell(b, b.pid_tmp + sb, sb, n, lane, 0, n, c0 + (uint32_t)k);
    else
      canon_large(b, b.pid_tmp + sb, sb, n, lane, c0 + (uint32_t)k);
  }
}

// ---- two-kernel build ------------------------------------------------------

constexpr int kTileShift = 6;  // 64 cells per k_canon_tiles block
constexpr int kTileThreads = 256;
constexpr int kCanonPer = 1;   // staged slots a k_canon_tiles thread loads at once (1
                               // measured fastest: 41.6 us, against 42.1 us for 2, 45.9 us for 4)

// Shared memory of a k_canon_tiles block staging up to `atoms` members:
// particle id, order key and local cell of each, after the fixed part.
__host__ __device__ constexpr uint32_t tile_smem(uint32_t atoms) { return atoms * 9u; }

// Atoms per thread of k_bin_buckets: a warp takes kBinPer groups of 32
// consecutive atoms and issues each dependent step (position, column rank,
// ticket) for all groups before the next.  On the B200 one group per warp
// and more resident warps measured fastest (41.6 us against 42.9 us for two
// groups at 1M atoms, cell build in the step).
constexpr int kBinPer = 1;

__global__ void __launch_bounds__(kTileThreads) k_bin_buckets(CellBufs b) {
  pdl_enter();
  const int lane = threadIdx.x & 31;
  const uint32_t w0 = (blockIdx.x * kTileThreads + (threadIdx.x & ~31u)) * kBinPer;
  uint32_t key[kBinPer], col[kBinPer], d2[kBinPer], sysi[kBinPer];
  float4 p[kBinPer];
#pragma unroll
  for (int k = 0; k < kBinPer; ++k) {
    const uint32_t i = w0 + 32u * k + lane;
    if (i < b.N) {
      p[k] = b.r[i];
      sysi[k] = system_of(b, i);
    }
  }
#pragma unroll
  for (int k = 0; k < kBinPer; ++k) {
    const uint32_t i = w0 + 32u * k + lane;
    col[k] = kNone;
    if (i < b.N) {
      const SysDesc &S = b.sys[sysi[k]];
      const int c0 = cell_coord(p[k].x, S.g.lo[0], S.g.len[0], S.g.n[0]);
      const int c1 = cell_coord(p[k].y, S.g.lo[1], S.g.len[1], S.g.n[1]);
      d2[k] = (uint32_t)cell_coord(p[k].z, S.g.lo[2], S.g.len[2], S.g.n[2]);
      col[k] = b.colrank[S.col0 + c0 * S.g.n[1] + c1];
    }
  }
#pragma unroll
  for (int k = 0; k < kBinPer; ++k) {
    const uint32_t i = w0 + 32u * k + lane;
    key[k] = kNone;
    if (i < b.N) {
      const SysDesc &S = b.sys[sysi[k]];
      key[k] = S.cell0 + col[k] * (uint32_t)S.g.n[2] + d2[k];
      b.key[i] = key[k];
    }
  }
  // tickets: one atomic per distinct cell of a group, its lanes ranked after it
  uint32_t peers[kBinPer], first[kBinPer];
#pragma unroll
  for (int k = 0; k < kBinPer; ++k) {
    peers[k] = __match_any_sync(0xffffffffu, key[k]);
    first[k] = 0;
    if (key[k] != kNone && __ffs(peers[k]) - 1 == lane)
      first[k] = atomicAdd(&b.count[key[k]], (uint32_t)__popc(peers[k]));
  }
#pragma unroll
  for (int k = 0; k < kBinPer; ++k) {
    const uint32_t f = __shfl_sync(0xffffffffu, first[k], __ffs(peers[k]) - 1);
    const uint32_t i = w0 + 32u * k + lane;
    if (key[k] == kNone) continue;
    const uint32_t t = f + (uint32_t)__popc(peers[k] & ((1u << lane) - 1u));
    if (t < b.bucket_cap) {
      b.bucket[(size_t)key[k] * b.bucket_cap + t] = i;
    } else {
      // at most N members overflow, so the list never does
      const uint32_t o = atomicAdd(&b.ctl[0], 1u);
      b.ovf[o] = make_uint2(key[k], i);
    }
  }
  // tile totals: one atomic per distinct tile of a group
#pragma unroll
  for (int k = 0; k < kBinPer; ++k) {
    const uint32_t tile = key[k] == kNone ? kNone : key[k] >> kTileShift;
    const uint32_t tp = __match_any_sync(0xffffffffu, tile);
    if (tile != kNone && __ffs(tp) - 1 == lane) atomicAdd(&b.tcount[tile], (uint32_t)__popc(tp));
  }
}

// The members of an overflowing cell (more than bucket_cap): the bucket, then
// its overflow entries in list order, gathered into pid_tmp[s0 ..); returns
// the member array.  Whole warp.
__device__ const uint32_t *gather_overflow(const CellBufs &b, uint32_t key, uint32_t s0,
                                           int lane) {
  uint32_t *dst = b.pid_tmp + s0;
  const uint32_t cap = b.bucket_cap;
  for (uint32_t a = lane; a < cap; a += 32) dst[a] = b.bucket[(size_t)key * cap + a];
  const uint32_t novf = b.ctl[0];
  uint32_t m = cap;
  for (uint32_t base = 0; base < novf; base += 32) {
    const uint2 e = base + lane < novf ? b.ovf[base + lane] : make_uint2(kNone, 0u);
    const bool mine = e.x == key;
    const uint32_t bal = __ballot_sync(0xffffffffu, mine);
    if (mine) dst[m + __popc(bal & ((1u << lane) - 1u))] = e.y;
    m += __popc(bal);
  }
  __syncwarp();
  return dst;
}

// Members of a cell that fits its bucket.
__device__ __forceinline__ const uint32_t *members(const CellBufs &b, uint32_t key) {
  return b.bucket + (size_t)key * b.bucket_cap;
}

// One block per 64-cell tile.  The tile's first slot is the sum of the tile
// counts before it (no block waits for another); the cells' starts follow
// from a scan of their counts.  A tile of at most tile_atoms members whose
// cells all fit their buckets is staged in shared memory: every thread
// gathers members (id, order key, cell) with independent loads, then ranks
// its members within their cells and writes them.  Other tiles take one
// warp per two cells.
__global__ void __launch_bounds__(kTileThreads, 8) k_canon_tiles(CellBufs b) {
  pdl_enter();
  extern __shared__ __align__(16) unsigned char tsm[];
  __shared__ uint32_t red[kTileThreads / 32];
  __shared__ uint32_t cst[(1 << kTileShift) + 1];  // tile-local starts, then the total
  __shared__ uint32_t wtot, nmax;
  __shared__ bool is_last;
  const uint32_t t = blockIdx.x, c0 = t << kTileShift;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t acc = 0;
  for (uint32_t k = threadIdx.x; k < t; k += kTileThreads) acc += b.tcount[k];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) red[warp] = acc;
  if (threadIdx.x == 0) nmax = 0;
  // counts of the tile's cells, scanned by warps 0 and 1
  uint32_t n = 0, incl = 0;
  const uint32_t c = c0 + threadIdx.x;
  if (threadIdx.x < (1u << kTileShift)) {
    n = c < b.ncells ? b.count[c] : 0u;
    incl = n;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
  }
  if (threadIdx.x == 31) wtot = incl;  // warp 0's total
  __syncthreads();
  uint32_t base = 0;
#pragma unroll
  for (int w = 0; w < kTileThreads / 32; ++w) base += red[w];
  if (threadIdx.x < (1u << kTileShift)) {
    const uint32_t loc = (warp == 1 ? wtot : 0u) + incl - n;
    cst[threadIdx.x] = loc;
    if (c < b.ncells) {
      b.start[c] = base + loc;
      b.count[c] = 0u;
      if (c == b.ncells - 1) b.start[b.ncells] = base + loc + n;
    }
    if (threadIdx.x == (1u << kTileShift) - 1) cst[1u << kTileShift] = loc + n;
    if (n > 0) atomicMax(&nmax, n);
  }
  __syncthreads();
  const uint32_t T = cst[1u << kTileShift];
  if (T <= b.tile_atoms && nmax <= b.bucket_cap) {
    uint32_t *sid = reinterpret_cast<uint32_t *>(tsm);
    uint32_t *szk = sid + b.tile_atoms;
    uint8_t *scl = reinterpret_cast<uint8_t *>(szk + b.tile_atoms);
    // gather: slot j of the tile -> (cell k, member j - cst[k]); a thread's
    // slots are taken kCanonPer at a time, each load step issued for all
    for (uint32_t j0 = threadIdx.x; j0 < T; j0 += kCanonPer * kTileThreads) {
      uint32_t me[kCanonPer];
#pragma unroll
      for (int u = 0; u < kCanonPer; ++u) {
        const uint32_t j = j0 + (uint32_t)u * kTileThreads;
        if (j >= T) break;
        uint32_t lo = 0, hi = 1u << kTileShift;  // largest k with cst[k] <= j
        while (hi - lo > 1) {
          const uint32_t mid = (lo + hi) >> 1;
          if (cst[mid] <= j) lo = mid; else hi = mid;
        }
        me[u] = members(b, c0 + lo)[j - cst[lo]];
        scl[j] = (uint8_t)lo;
      }
#pragma unroll
      for (int u = 0; u < kCanonPer; ++u) {
        const uint32_t j = j0 + (uint32_t)u * kTileThreads;
        if (j >= T) break;
        sid[j] = me[u];
        szk[j] = z_key(b.r[me[u]].z);
      }
    }
    __syncthreads();
    // rank within the cell by (z, particle id), then write
    for (uint32_t j0 = threadIdx.x; j0 < T; j0 += kCanonPer * kTileThreads) {
      float4 p[kCanonPer];
      uint32_t ty[kCanonPer], sy[kCanonPer];
#pragma unroll
      for (int u = 0; u < kCanonPer; ++u) {
        const uint32_t j = j0 + (uint32_t)u * kTileThreads;
        if (j >= T) break;
        const uint32_t me = sid[j];
        p[u] = b.r[me];
        ty[u] = b.type[me];
        sy[u] = system_of(b, me);
      }
#pragma unroll
      for (int u = 0; u < kCanonPer; ++u) {
        const uint32_t j = j0 + (uint32_t)u * kTileThreads;
        if (j >= T) break;
        const uint32_t k = scl[j], lo = cst[k], hi = cst[k + 1];
        const uint32_t me = sid[j], kz = szk[j];
        uint32_t rank = 0;
        for (uint32_t q = lo; q < hi; ++q) rank += canon_before(szk[q], sid[q], kz, me) ? 1u : 0u;
        const uint32_t s = base + lo + rank;
        b.pid[s] = me;
        b.slot[me] = s;
        b.rs[s] = make_float4(p[u].x, p[u].y, p[u].z, __int_as_float((int)ty[u]));
        if (b.xs) write_mirror_of(b, b.sys[sy[u]], s, p[u], c0 + k, ty[u]);
      }
    }
  } else {
    // one warp per two cells, 16 cells per round
    for (uint32_t r = 0; r < (1u << kTileShift); r += 2 * (kTileThreads / 32)) {
      const uint32_t k0 = r + 2 * (uint32_t)warp;
      const uint32_t ca = c0 + k0;
      if (ca >= b.ncells) break;
      const bool two = ca + 1 < b.ncells;
      const uint32_t s0 = base + cst[k0], s1 = base + cst[k0 + 1];
      const uint32_t s2 = two ? base + cst[k0 + 2] : s1;
      const uint32_t n0 = s1 - s0, n1 = s2 - s1;
      if (n0 <= 16 && n1 <= 16) {
        const int half = lane >> 4;
        const uint32_t key = ca + (uint32_t)half;
        canon_cell(b, members(b, key), half ? s1 : s0, half ? n1 : n0, lane & 15, half * 16,
                   max(n0, n1), key);
        continue;
      }
      for (int k = 0; k < (two ? 2 : 1); ++k) {
        const uint32_t sb = k ? s1 : s0, nn = k ? n1 : n0, key = ca + (uint32_t)k;
        if (nn <= 32)
          canon_cell(b, members(b, key), sb, nn, lane, 0, nn, key);
        else if (nn <= b.bucket_cap)
          canon_large(b, members(b, key), sb, nn, lane, key);
        else
          canon_large(b, gather_overflow(b, key, sb, lane), sb, nn, lane, key);
      }
    }
  }
  // the last block to finish clears the tile and overflow counts for the next
  // build (every block has read them by then)
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    is_last = atomicAdd(&b.ctl[1], 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (is_last) {
    for (uint32_t k = threadIdx.x; k < b.ntile; k += kTileThreads) b.tcount[k] = 0u;
    if (threadIdx.x == 0) {
      b.ctl[0] = 0u;
      b.ctl[1] = 0u;
    }
  }
}

}  // namespace

cudaError_t launch_cell_build(const CellBufs &b, cudaStream_t s) {
  if (b.N == 0) return cudaSuccess;
  const uint32_t nb = (b.N + 255) / 256;
  if (b.bucket != nullptr) {
    const uint32_t per_block = kTileThreads * kBinPer;
    cudaError_t e = launch_pdl(k_bin_buckets, dim3((b.N + per_block - 1) / per_block),
                               dim3(kTileThreads), 0, s, b);
    const uint32_t smem = tile_smem(b.tile_atoms);
    if (e == cudaSuccess && smem > 48u * 1024u)
      e = cudaFuncSetAttribute(k_canon_tiles, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)smem);
    if (e == cudaSuccess)
      e = launch_pdl(k_canon_tiles, dim3(b.ntile), dim3(kTileThreads), smem, s, b);
    return e;
  }
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
