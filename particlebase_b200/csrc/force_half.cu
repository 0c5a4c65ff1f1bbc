// Lennard-Jones pair forces over the cell list, each pair computed once.
//
// Same physics as the full-shell kernel (force.cu) and the reference's
// cudaParticleMD::calcForce (cudaParticleMD.cu:24-69, calcF_IJpairWithBlock_F4
// with MDpairForce<potentialLJ>, kerneltemplate.hh:229-294, 523-565,
// kernelinline.hh:86-96): truncated, unshifted LJ over the 27-cell stencil
// with the minimum image.  The reference evaluates every ordered pair; here
// every unordered pair is evaluated once and its force is added to both atoms
// (Newton's third law), which halves the candidate tests and the force
// evaluations.
//
// Half shell.  A work item is (system, x-y column, run of z cells [z0, z1)),
// as in force.cu, but it stages only 5 of the 9 neighbour columns: the home
// column and the 4 "forward" ones at x-y offsets (0, +1), (+1, -1), (+1, 0),
// (+1, +1).  A pair whose partner sits in a forward column belongs to the
// item of the home atom; its mirror image (the partner's item) would see the
// home column as a backward neighbour, which it does not stage.  In the home
// column a pair belongs to the item of the atom that comes first in the
// staged (frame z, particle id) order, so the partner must come later: the
// home column is staged first, and the rule is "staged slot of j > staged
// slot of i".  With cells at least rc wide, every pair within the cutoff is
// found through exactly one image, so every pair is counted exactly once.
//
// Deterministic sums.  The force on an atom is the sum of its own (i-side)
// share and the partner (j-side) shares that other clusters, warps, CTAs and
// items add to it, in an order that changes from run to run.  Every share is
// therefore rounded once to a fixed-point integer with 32 fractional bits
// (resolution 2.3e-10) and added with integer atomics, which are exact and
// order-independent: the sums, and every result downstream, are the same bits
// in every run and whether a system runs alone or in a batch.  A consumer
// warp adds its j-side shares, and its home atoms' i-side sums once per
// cluster, to per-slot accumulators of the stage buffer in shared memory:
// each 64-bit share c is split into c >> 20 and its low 20 bits, added with
// native 32-bit atomics (red.shared.add.u32) to two words whose combination
// hi 2^20 + lo is exact for the sums an item can produce (below).  When the
// consumers release the buffer, the producer warps add every staged atom's
// accumulator to a global 64-bit fixed-point array indexed by sorted slot
// (red.global.add.u64) and clear it.  k_force_finish
// turns the global sums into FP32 forces in particle order and clears them for
// the next call.
//
// Range.  A stage accumulator takes shares below 2^11 in magnitude: the hi
// word then holds sums up to 2^19, more than 250 such shares, while an atom
// has fewer than 100 partners inside the cutoff at any liquid density, and
// the lo word holds 4,096 shares.  Larger shares go straight to the global
// sums: the fine one (2^-32 units) below 2^22, where even 500 shares stay
// inside 64 bits, and a coarse one in units of 1/2 up to 2^62 (every FP32
// value of that magnitude is a multiple of 1/2, so these are exact too) for
// atoms pressed far inside each other, which MD states do not reach but random
// starts can.  A NaN share, or one beyond 2^62, is dropped and raises
// PB_STATUS_NONFINITE.
//
// Energies count each pair once (u, u - U(rc), f r^2) and the pair counter
// advances by 2, so the totals equal the full-shell kernel's halved sums.
#include <algorithm>

#include "force_common.cuh"
#include "integrate.cuh"

namespace pb {
namespace {

constexpr int kCols = 5;       // staged columns: the home column, then its 4 forward neighbours
constexpr int kRuns = 3 * kCols;
constexpr float kFix = 4294967296.0f;        // 2^32: fixed-point scale of the force sums
constexpr float kStage = 2048.0f;            // 2^11: largest share of the stage accumulators
constexpr float kSmall = 4194304.0f;         // 2^22: largest share of the fine sums
constexpr float kHuge = 4.611686018427388e18f; // 2^62: largest share of the coarse sums

// Index of staged column c in the 3 x 3 neighbour table of a work item
// (x offset outer, y offset inner, each -1, 0, +1): the home column (0, 0) is
// entry 4, and (0, +1), (+1, -1), (+1, 0), (+1, +1) are entries 5 .. 8.
__host__ __device__ __forceinline__ int nb9(int c) { return 4 + c; }

// One work item as the consumers see it (written by the producers).
template <int NT>
struct ItemDesc3 {
  uint32_t off[kCols][kMaxSeg + 3];  // as ItemDesc in force.cu, for 5 columns
  uint32_t ps[kCols + 1];
  uint32_t kbase[kCols];
  float sx[kCols], sy[kCols];
  float sz_lo, sz_mid, sz_hi;
  uint32_t item, sys, home_g0, hb, H, nclus, ntask, sentinel, base;
  int z0, nz, nseg;
  int skip;
  int overflow;
  LJLocal<NT> lj;
  uint16_t q0[kWinCap][kCols], len[kWinCap][kCols], pre[kWinCap][kCols];
  uint16_t Q[kWinCap], M[kWinCap];
  // copy run p of the stage: stage slot of its first real atom, its real
  // atoms, and the sorted slot of that atom (the accumulator flush map)
  uint32_t run_s[kRuns], run_n[kRuns], run_g[kRuns];
};

struct Scratch3 {
  uint32_t gstart[kCols][kMaxSeg + 3];
  uint32_t cnt[kCols][kMaxSeg + 3];
  uint32_t dst[kRuns], lead[kRuns], n[kRuns], alen[kRuns];
  float shift[kRuns][3];
  uint32_t shifted;
};

// One stage buffer: coordinate planes and the fixed-point accumulators.
struct Stage {
  float *X, *Y, *Z;
  uint32_t *T;
  uint32_t *A;  // 6 planes of `slots` words: hi x, y, z, then lo x, y, z
  uint32_t slots;
};

// Slots for `cap` staged atoms: up to 3 copy runs per column, each bringing at
// most 6 neighbouring atoms along, plus the quad of far atoms.
__host__ __device__ __forceinline__ uint32_t padded_slots3(uint32_t cap) {
  return ((cap + 6u * kRuns + 3u) & ~3u) + 4u;
}

__host__ __device__ __forceinline__ uint32_t plane_bytes3(uint32_t slots, int nt) {
  return (slots * (nt > 1 ? 16u : 12u) + 15u) & ~15u;
}

__host__ __device__ __forceinline__ uint32_t stage_bytes3(uint32_t slots, int nt) {
  return plane_bytes3(slots, nt) + 24u * slots;
}

__host__ __device__ __forceinline__ uint32_t warp_bytes3(uint32_t slots) {
  return ((32u * kListLen * 2u + (slots / 4u + kChunk) * 2u) + 15u) & ~15u;
}

__host__ __device__ __forceinline__ uint32_t smem_bytes3(uint32_t cap, int consumers, int nt) {
  const uint32_t slots = padded_slots3(cap);
  return 2u * stage_bytes3(slots, nt) + (uint32_t)consumers * warp_bytes3(slots);
}

__device__ __forceinline__ void red_shared_u32(uint32_t addr, uint32_t v) {
  asm volatile("red.shared.add.u32 [%0], %1;" ::"r"(addr), "r"(v) : "memory");
}

__device__ __forceinline__ void red_global_u64(unsigned long long *p, long long v) {
  asm volatile("red.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// A force share in the fine fixed point: round(v 2^32), |v| < 2^22.
__device__ __forceinline__ long long fix32(float v) { return __float2ll_rn(v * kFix); }

// A share of any size for the atom at sorted slot g, straight to the global
// sums: the fine sum below 2^22, the coarse one (units of 1/2) up to 2^62;
// NaN and larger shares are dropped and recorded in `bad`.
__device__ __forceinline__ void share_global(const ForceBufs &b, uint32_t g, int c, float v,
                                             bool &bad) {
  const float a = fabsf(v);
  if (a < kSmall) {
    red_global_u64(b.facc + (size_t)c * b.nacc + g, fix32(v));
  } else if (a < kHuge) {
    red_global_u64(b.fbig + (size_t)c * b.nacc + g, __float2ll_rn(v * 2.0f));
  } else {
    bad = true;
  }
}

// Add the share (x, y, z), each below 2^11, to the accumulator of stage slot
// s: c = round(v 2^32) goes in as c >> 20 (hi word) and c & (2^20 - 1) (lo).
// `abase` is the shared address of the hi x plane, `pstride` the plane size
// in bytes.
__device__ __forceinline__ void stage_add3(uint32_t abase, uint32_t pstride, uint32_t s, float x,
                                           float y, float z) {
  const float v[3] = {x, y, z};
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const long long q = fix32(v[c]);
    red_shared_u32(abase + c * pstride + 4u * s, (uint32_t)(int)(q >> 20));
    red_shared_u32(abase + (3 + c) * pstride + 4u * s, (uint32_t)q & 0xfffffu);
  }
}

// Largest magnitude of three components.
__device__ __forceinline__ float max3abs(float x, float y, float z) {
  return fmaxf(fabsf(x), fmaxf(fabsf(y), fabsf(z)));
}

// ---- producer ---------------------------------------------------------------

template <int NT, int kProd>
__device__ bool produce_item3(const ForceBufs &b, uint32_t item, ItemDesc3<NT> &d, Scratch3 &sc,
                              const Stage &pl, uint64_t *landed, uint32_t &lphase,
                              uint32_t &running, int kCons) {
  constexpr int kPT = kProd * 32;
  const int pt = threadIdx.x, lane = pt & 31, pw = pt >> 5;
  const ForceItem it = b.items[item];
  const bool skip = b.steps_left != nullptr && b.steps_left[it.sys] == 0;
  if (pt == 0) {
    d.item = item;
    d.sys = it.sys;
    d.skip = skip;
    d.overflow = 0;
    d.H = 0;
    d.nclus = 0;
    d.ntask = 0;
  }
  if (skip) {
    producer_sync<kProd>();
    return true;
  }
  const SysDesc &S = b.sys[it.sys];
  const Grid g = S.g;
  const uint32_t mirror0 = S.mirror0, atom0 = S.atom0, scap = S.cap_half;
  const int nx = g.n[0], ny = g.n[1], nz = g.n[2];
  const int z0 = it.z0, z1 = it.z1, nseg = z1 - z0;
  const int ncell = nseg + 2;
  for (int t = pt; t < NT * NT; t += kPT) {
    const LJTable &Tb = b.lj[S.lj];
    const int a = t / NT, c = t % NT;
    const int k = a * Tb.nt + c;
    d.lj.s2[t] = Tb.s2[k];
    d.lj.e24[t] = Tb.e24[k];
    d.lj.e4[t] = Tb.e4[k];
    d.lj.rc2[t] = Tb.rc2[k];
    d.lj.ush[t] = Tb.ushift[k];
  }
  if (pt < kCols) {
    const int c = pt, k9 = nb9(c);
    const int ax = it.cx + k9 / 3 - 1, ay = it.cy + k9 % 3 - 1;
    const int wx = ax < 0 ? -1 : (ax >= nx ? 1 : 0);
    const int wy = ay < 0 ? -1 : (ay >= ny ? 1 : 0);
    const float Fx = it.cx == nx - 1 ? g.L[0] : 0.0f, Fy = it.cy == ny - 1 ? g.L[1] : 0.0f;
    d.sx[c] = Fx - (float)wx * g.L[0];
    d.sy[c] = Fy - (float)wy * g.L[1];
    d.kbase[c] = it.kbase[k9];
  }
  // an item on the top face works in the frame shifted down by L, where the
  // shifts of its atoms (all in the upper half) are exact; a whole column
  // keeps the unshifted frame and rounds only the image above its top
  const float Fz = z1 == nz && z0 > 0 ? g.L[2] : 0.0f;
  const float sz_lo = z0 == 0 ? Fz + g.L[2] : Fz;
  const float sz_hi = z1 == nz ? Fz - g.L[2] : Fz;
  if (pt == 0) {
    d.sz_lo = sz_lo;
    d.sz_mid = Fz;
    d.sz_hi = sz_hi;
    d.z0 = z0;
    d.nz = nz;
    d.nseg = nseg;
  }
  for (int t = pt; t < kCols * ncell; t += kPT) {
    const int c = t / ncell, k = t % ncell;
    const int zc = (z0 - 1 + k + nz) % nz;
    const uint32_t key = it.kbase[nb9(c)] + (uint32_t)zc;
    const uint32_t s0 = b.start[key];
    sc.gstart[c][k] = s0;
    sc.cnt[c][k] = b.start[key + 1] - s0;
  }
  producer_sync<kProd>();
  for (int c = pw; c < kCols; c += kProd) {
    uint32_t run = 0;
    for (int base = 0; base < ncell; base += 32) {
      const int k = base + lane;
      const uint32_t v = k < ncell ? sc.cnt[c][k] : 0u;
      uint32_t incl = v;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
      }
      if (k < ncell) d.off[c][k] = run + incl - v;
      run += __shfl_sync(0xffffffffu, incl, 31);
    }
    if (lane == 0) d.off[c][ncell] = run;
  }
  producer_sync<kProd>();
  const int a_end = z0 == 0 ? 1 : 0, c_beg = z1 == nz ? ncell - 1 : ncell;
  const uint32_t H = d.off[0][nseg + 1] - d.off[0][1];
  const uint32_t nclus = (H + 7) / 8;
  if (pw == 0) {
    uint32_t n = 0, m0 = 0, ma = 0, alen = 0, g0 = 0;
    if (lane < kRuns) {
      const int c = lane / 3, p = lane % 3;
      const int k0 = p == 0 ? 0 : (p == 1 ? a_end : c_beg);
      const int k1 = p == 0 ? a_end : (p == 1 ? c_beg : ncell);
      n = d.off[c][k1] - d.off[c][k0];
      if (n > 0) {
        g0 = sc.gstart[c][k0];
        m0 = mirror0 + (g0 - atom0);
        ma = m0 & ~3u;
        alen = ((m0 + n + 3u) & ~3u) - ma;
      }
    }
    uint32_t incl = alen;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    const uint32_t dst = incl - alen;
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    float rx = 0.f, ry = 0.f, rz = 0.f;
    if (lane < kRuns) {
      const int c = lane / 3, pp = lane % 3;
      rx = d.sx[c];
      ry = d.sy[c];
      rz = pp == 0 ? sz_lo : (pp == 1 ? Fz : sz_hi);
      sc.dst[lane] = dst;
      sc.lead[lane] = m0 - ma;
      sc.n[lane] = n;
      sc.alen[lane] = alen;
      sc.shift[lane][0] = rx;
      sc.shift[lane][1] = ry;
      sc.shift[lane][2] = rz;
      d.run_s[lane] = dst + (m0 - ma);
      d.run_n[lane] = n;
      d.run_g[lane] = g0;
      if (lane % 3 == 0) d.ps[lane / 3] = dst;
    }
    const uint32_t shifted =
        __ballot_sync(0xffffffffu, n > 0 && (rx != 0.f || ry != 0.f || rz != 0.f));
    if (lane == 0) sc.shifted = shifted;
    const bool overflow = total + 4u > padded_slots3(scap) || nclus > (uint32_t)kWinCap;
    if (lane == 0) {
      d.ps[kCols] = total;
      d.H = H;
      d.home_g0 = sc.gstart[0][1];
      d.overflow = overflow;
      if (overflow) {
        d.ntask = min((H + 31) / 32, (uint32_t)kWinCap);
        atomicOr(&b.status[it.sys], kStatusSmemOverflow);
      }
    }
    if (!overflow && total > 0) {
      uint32_t bytes = alen * 4u * (NT > 1 ? 4u : 3u);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) bytes += __shfl_xor_sync(0xffffffffu, bytes, o);
      if (lane == 0) mbar_arrive_expect_tx(landed, bytes);
      __syncwarp();
      if (lane < kRuns && alen > 0) {
        bulk_g2s(pl.X + dst, b.xs + ma, alen * 4u, landed);
        bulk_g2s(pl.Y + dst, b.ys + ma, alen * 4u, landed);
        bulk_g2s(pl.Z + dst, b.zs + ma, alen * 4u, landed);
        if (NT > 1) bulk_g2s(pl.T + dst, b.ts + ma, alen * 4u, landed);
      }
    }
  }
  producer_sync<kProd>();
  if (d.overflow) return true;
  const uint32_t total = d.ps[kCols];
  if (total > 0) {
    bool ok = pt != 0 || mbar_wait_or_abort(landed, lphase, &kNeverAbort);
    lphase ^= 1u;
    if (pt == 0 && !ok) {
      atomicOr(&b.status[it.sys], kStatusWaitTimeout);
      mbar_wait_bounded(landed, lphase ^ 1u);
      d.skip = 2;
    }
    producer_sync<kProd>();
    if (d.skip == 2) return false;
    for (uint32_t m = sc.shifted; m != 0u; m &= m - 1u) {
      const int p = __ffs(m) - 1;
      const float sx = sc.shift[p][0], sy = sc.shift[p][1], sz = sc.shift[p][2];
      const uint32_t s0 = sc.dst[p] + sc.lead[p], s1 = s0 + sc.n[p];
      for (uint32_t s = s0 + pt; s < s1; s += kPT) {
        pl.X[s] -= sx;
        pl.Y[s] -= sy;
        pl.Z[s] -= sz;
      }
    }
    producer_sync<kProd>();
    if (pt < kRuns && sc.alen[pt] > 0) {
      const uint32_t dst = sc.dst[pt], s0 = dst + sc.lead[pt], s1 = s0 + sc.n[pt];
      const float zlo = pl.Z[s0], zhi = pl.Z[s1 - 1];
      for (uint32_t s = dst; s < s0; ++s) {
        pl.X[s] = kFar;
        pl.Y[s] = kFar;
        pl.Z[s] = zlo;
        if (NT > 1) pl.T[s] = 0u;
      }
      for (uint32_t s = s1; s < dst + sc.alen[pt]; ++s) {
        pl.X[s] = kFar;
        pl.Y[s] = kFar;
        pl.Z[s] = zhi;
        if (NT > 1) pl.T[s] = 0u;
      }
    }
  }
  if (pt >= 32 * (kProd - 1) && pt < 32 * (kProd - 1) + 4) {
    const uint32_t s = total + (uint32_t)(pt - 32 * (kProd - 1));
    pl.X[s] = kFar;
    pl.Y[s] = kFar;
    pl.Z[s] = kFar;
    if (NT > 1) pl.T[s] = 0u;
  }
  producer_sync<kProd>();
  // z windows of every (cluster, column).  In the home column a cluster's
  // partners come after its first atom, so its window starts there.
  const int hp = 1;  // run of the home column that holds home cells 1 .. nseg
  const uint32_t hb = sc.dst[hp] + sc.lead[hp] + (d.off[0][1] - d.off[0][a_end]);
  float rcmax2 = 0.f;
  for (int k = 0; k < NT * NT; ++k) rcmax2 = fmaxf(rcmax2, d.lj.rc2[k]);
  const float rcw = sqrtf(rcmax2) * 1.00001f + 1e-5f;
  for (uint32_t t = pt; t < (uint32_t)kCols * nclus; t += kPT) {
    const uint32_t k = t / kCols, c = t - kCols * k;
    const float zmin = pl.Z[hb + k * 8];
    const float zmax = pl.Z[hb + min(k * 8 + 7, H - 1)];
    const uint32_t lo = d.ps[c], hi = d.ps[c + 1];
    const uint32_t a = c == 0 ? (hb + k * 8) >> 2 : lower_bound_z(pl.Z, lo, hi, zmin - rcw) >> 2;
    const uint32_t e = (upper_bound_z(pl.Z, lo, hi, zmax + rcw) + 3u) >> 2;
    d.q0[k][c] = (uint16_t)a;
    d.len[k][c] = (uint16_t)(e > a ? e - a : 0u);
  }
  producer_sync<kProd>();
  for (uint32_t k = pt; k < nclus; k += kPT) {
    uint32_t s = 0, m = 2;
    for (int c = 0; c < kCols; ++c) {
      d.pre[k][c] = (uint16_t)s;
      s += d.len[k][c];
      m = max(m, (uint32_t)d.len[k][c]);
    }
    d.Q[k] = (uint16_t)s;
    d.M[k] = (uint16_t)m;
  }
  if (pt == 0) {
    d.hb = hb;
    d.nclus = nclus;
    d.sentinel = total / 4u;
    d.base = running % (uint32_t)kCons;
  }
  running += nclus;
  producer_sync<kProd>();
  return true;
}

// Producers: add a released buffer's accumulators to the global sums, clear
// them, and write the item's energy partials.
template <int NT, int kProd, bool ENERGY>
__device__ void retire_item3(const ForceBufs &b, const ItemDesc3<NT> &d, const Stage &pl,
                             const double (*e)[4]) {
  constexpr int kPT = kProd * 32;
  const int pt = threadIdx.x;
  if (!d.skip && !d.overflow) {
    const size_t n3 = b.nacc;
    for (int p = 0; p < kRuns; ++p) {
      const uint32_t s0 = d.run_s[p], n = d.run_n[p], g0 = d.run_g[p];
      for (uint32_t k = pt; k < n; k += kPT) {
        const uint32_t s = s0 + k;
        unsigned long long *acc = b.facc + g0 + k;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const int hi = (int)pl.A[c * pl.slots + s];
          const uint32_t lo = pl.A[(3 + c) * pl.slots + s];
          const long long v = (long long)hi * 1048576ll + (long long)lo;
          if (v != 0) red_global_u64(acc + c * n3, v);
          pl.A[c * pl.slots + s] = 0u;
          pl.A[(3 + c) * pl.slots + s] = 0u;
        }
      }
    }
  }
  if (ENERGY && pt == 0) {
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    if (!d.skip) {
      const uint32_t n = d.overflow ? d.ntask : d.nclus;
      for (uint32_t k = 0; k < n; ++k)
        for (int c = 0; c < 4; ++c) v[c] += e[k][c];
    }
    for (int c = 0; c < 4; ++c) b.partials[(size_t)d.item * 4 + c] = v[c];
  }
}

// ---- consumers --------------------------------------------------------------

// Phase 2: the listed pairs of this lane, two per step in packed FP32x2.  A
// pair counts when it lies inside the exact cutoff of its types, comes later
// than the home atom in the staged order (j > hs) and is not coincident; its
// force is added to the lane's i-side sums and, in fixed point, to the
// partner's accumulator.
template <int NT, bool ENERGY, typename GSlot>
__device__ __forceinline__ void flush_half(const ForceBufs &b, const Stage &pl,
                                           const uint16_t *list, uint32_t cnt, int lane,
                                           uint32_t hs, float xi, float yi, float zi, int ti,
                                           const LJLocal<NT> &lj, GSlot gslot, float2 (&f3)[3],
                                           float2 (&en)[3], uint32_t &npair, bool &bad) {
  const float2 m1 = make_float2(-1.0f, -1.0f);
  const float2 xi2 = make_float2(xi, xi), yi2 = make_float2(yi, yi), zi2 = make_float2(zi, zi);
  const float2 two = make_float2(2.0f, 2.0f), mone = make_float2(-1.0f, -1.0f);
  float2 s2 = make_float2(lj.s2[0], lj.s2[0]), e24 = make_float2(lj.e24[0], lj.e24[0]);
  float2 e4 = make_float2(lj.e4[0], lj.e4[0]), ush = make_float2(lj.ush[0], lj.ush[0]);
  float rc2a = lj.rc2[0], rc2b = lj.rc2[0];
  const uint32_t xa = smem_u32(pl.X), ya = smem_u32(pl.Y), za = smem_u32(pl.Z);
  const uint32_t aa = smem_u32(pl.A), astride = 4u * pl.slots;
  const uint32_t la = smem_u32(list) + 2u * (uint32_t)lane;
  for (uint32_t k = 0; k < cnt; k += 2) {
    const uint32_t j0 = lds_u16(la + 64u * k);
    const uint32_t j1 = lds_u16(la + 64u * min(k + 1, cnt - 1));
    const bool v1 = k + 1 < cnt;
    if (NT > 1) {
      const int ka = ti * NT + (int)pl.T[j0], kb = ti * NT + (int)pl.T[j1];
      s2 = make_float2(lj.s2[ka], lj.s2[kb]);
      e24 = make_float2(lj.e24[ka], lj.e24[kb]);
      rc2a = lj.rc2[ka];
      rc2b = lj.rc2[kb];
      if (ENERGY) {
        e4 = make_float2(lj.e4[ka], lj.e4[kb]);
        ush = make_float2(lj.ush[ka], lj.ush[kb]);
      }
    }
    const float2 dx =
        __ffma2_rn(make_float2(lds_f32(xa + 4u * j0), lds_f32(xa + 4u * j1)), m1, xi2);
    const float2 dy =
        __ffma2_rn(make_float2(lds_f32(ya + 4u * j0), lds_f32(ya + 4u * j1)), m1, yi2);
    const float2 dz =
        __ffma2_rn(make_float2(lds_f32(za + 4u * j0), lds_f32(za + 4u * j1)), m1, zi2);
    const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
    const bool ina = r2.x < rc2a && r2.x > 0.0f && j0 > hs;
    const bool inb = v1 && r2.y < rc2b && r2.y > 0.0f && j1 > hs;
    const float2 inv = make_float2(rcp_approx(r2.x), rcp_approx(r2.y));
    const float2 sr2 = __fmul2_rn(s2, inv);
    const float2 sr6 = __fmul2_rn(__fmul2_rn(sr2, sr2), sr2);
    const float2 t = __ffma2_rn(two, sr6, mone);
    float2 f = __fmul2_rn(__fmul2_rn(__fmul2_rn(e24, sr6), t), inv);
    f.x = ina ? f.x : 0.0f;
    f.y = inb ? f.y : 0.0f;
    const float2 fx = __fmul2_rn(f, dx), fy = __fmul2_rn(f, dy), fz = __fmul2_rn(f, dz);
    f3[0] = __fadd2_rn(f3[0], fx);
    f3[1] = __fadd2_rn(f3[1], fy);
    f3[2] = __fadd2_rn(f3[2], fz);
    if (ina) {
      if (max3abs(fx.x, fy.x, fz.x) < kStage) {
        stage_add3(aa, astride, j0, -fx.x, -fy.x, -fz.x);
      } else {
        const uint32_t g = gslot(j0);
        share_global(b, g, 0, -fx.x, bad);
        share_global(b, g, 1, -fy.x, bad);
        share_global(b, g, 2, -fz.x, bad);
      }
    }
    if (inb) {
      if (max3abs(fx.y, fy.y, fz.y) < kStage) {
        stage_add3(aa, astride, j1, -fx.y, -fy.y, -fz.y);
      } else {
        const uint32_t g = gslot(j1);
        share_global(b, g, 0, -fx.y, bad);
        share_global(b, g, 1, -fy.y, bad);
        share_global(b, g, 2, -fz.y, bad);
      }
    }
    if (ENERGY) {
      float2 u = __fmul2_rn(__fmul2_rn(e4, sr6), __fadd2_rn(sr6, mone));
      u.x = ina ? u.x : 0.0f;
      u.y = inb ? u.y : 0.0f;
      float2 us = __fadd2_rn(u, make_float2(-ush.x, -ush.y));
      us.x = ina ? us.x : 0.0f;
      us.y = inb ? us.y : 0.0f;
      en[0] = __fadd2_rn(en[0], u);
      en[1] = __fadd2_rn(en[1], us);
      en[2] = __ffma2_rn(f, r2, en[2]);
      npair += 2u * ((uint32_t)ina + (uint32_t)inb);
    }
  }
}

template <int NT, bool ENERGY>
__device__ __forceinline__ void consume_cluster3(const ForceBufs &b, const ItemDesc3<NT> &d,
                                                 const Stage &pl, uint32_t cl, uint16_t *mylist,
                                                 uint16_t *tb, double (&ce)[4], bool &bad) {
  const int lane = threadIdx.x & 31;
  const int il = lane & 7, q = lane >> 3;
  const float *X = pl.X, *Y = pl.Y, *Z = pl.Z;
  const uint32_t H = d.H, hb = d.hb;
  const uint32_t h = cl * 8 + il;
  const bool valid = h < H;
  const uint32_t hs = hb + (valid ? h : H - 1);
  const float xi = valid ? X[hs] : kNoAtom;
  const float yi = valid ? Y[hs] : kNoAtom;
  const float zi = valid ? Z[hs] : kNoAtom;
  const int ti = NT == 1 ? 0 : (int)pl.T[hs];
  const uint32_t Q = d.Q[cl], M = d.M[cl];
  const uint32_t magic = 0xffffffffu / M + 1u;
  for (uint32_t idx = lane; idx < (uint32_t)kCols * M; idx += 32) {
    const uint32_t c = __umulhi(idx, magic), i = idx - c * M;
    if (i < d.len[cl][c]) tb[table_pos(d.pre[cl][c] + i)] = (uint16_t)(d.q0[cl][c] + i);
  }
  for (uint32_t u = Q + lane; u < ((Q + 15u) & ~15u); u += 32)
    tb[table_pos(u)] = (uint16_t)d.sentinel;
  __syncwarp();

  float rcmax2 = 0.f;
  for (int k = 0; k < NT * NT; ++k) rcmax2 = fmaxf(rcmax2, d.lj.rc2[k]);
  const float2 nrc = make_float2(-rcmax2 * (1.0f + 1.0f / 1024.0f),
                                 -rcmax2 * (1.0f + 1.0f / 1024.0f));
  const float2 m1 = make_float2(-1.0f, -1.0f);
  float2 f3[3] = {{0.f, 0.f}, {0.f, 0.f}, {0.f, 0.f}};
  float2 en[3] = {{0.f, 0.f}, {0.f, 0.f}, {0.f, 0.f}};
  uint32_t npair = 0;
  const uint32_t hsv = valid ? hs : 0xffffffffu;  // padded lanes count no pair
  // sorted slot of the atom at stage slot s (its copy run), for the rare
  // shares too large for the stage's fine sums
  auto gslot = [&](uint32_t s) -> uint32_t {
    for (int p = 0; p < kRuns; ++p)
      if (s - d.run_s[p] < d.run_n[p]) return d.run_g[p] + (s - d.run_s[p]);
    return 0u;  // not reached: only real atoms receive shares
  };
  auto flush = [&](uint32_t cnt) {
    flush_half<NT, ENERGY>(b, pl, mylist, cnt, lane, hsv, xi, yi, zi, ti, d.lj, gslot, f3, en,
                           npair, bad);
  };
  const float2 xi2 = make_float2(xi, xi), yi2 = make_float2(yi, yi), zi2 = make_float2(zi, zi);
  const uint32_t xa = smem_u32(X), ya = smem_u32(Y), za = smem_u32(Z);
  const uint32_t lbase = smem_u32(mylist) + 2u * (uint32_t)lane;
  uint32_t oa = lbase;
  for (uint32_t u0 = 0; u0 < Q; u0 += kChunk) {
    const uint32_t cnt = (oa - lbase) >> 6;
    if (__reduce_max_sync(0xffffffffu, cnt) > (uint32_t)(kListLen - kChunk)) {
      flush(cnt);
      __syncwarp();
      oa = lbase;
    }
    const uint2 qq = *reinterpret_cast<const uint2 *>(tb + u0 + 4 * q);
    const uint32_t quads[4] = {qq.x & 0xffffu, qq.x >> 16, qq.y & 0xffffu, qq.y >> 16};
    const uint32_t nsteps = min((Q - u0 + 3u) >> 2, (uint32_t)(kChunk / 4));
    // one quad: 4 candidate tests, appended through offsets that depend on
    // the hit bits only, so the list pointer carries one add per quad
    auto test_quad = [&](uint32_t quad) {
      const float4 x4 = lds_f4(xa + quad * 16u), y4 = lds_f4(ya + quad * 16u),
                   z4 = lds_f4(za + quad * 16u);
      const float2 dxa = __ffma2_rn(make_float2(x4.x, x4.y), m1, xi2);
      const float2 dxb = __ffma2_rn(make_float2(x4.z, x4.w), m1, xi2);
      const float2 dya = __ffma2_rn(make_float2(y4.x, y4.y), m1, yi2);
      const float2 dyb = __ffma2_rn(make_float2(y4.z, y4.w), m1, yi2);
      const float2 dza = __ffma2_rn(make_float2(z4.x, z4.y), m1, zi2);
      const float2 dzb = __ffma2_rn(make_float2(z4.z, z4.w), m1, zi2);
      const float2 da = __ffma2_rn(dza, dza, __ffma2_rn(dya, dya, __ffma2_rn(dxa, dxa, nrc)));
      const float2 db = __ffma2_rn(dzb, dzb, __ffma2_rn(dyb, dyb, __ffma2_rn(dxb, dxb, nrc)));
      // hit = sign bit of r^2 - rc^2 (1 + 2^-10); a -0 or NaN sign only admits a
      // candidate that phase 2's exact test then drops
      const uint32_t h0 = __float_as_uint(da.x) >> 31, h1 = __float_as_uint(da.y) >> 31;
      const uint32_t h2 = __float_as_uint(db.x) >> 31, h3 = __float_as_uint(db.y) >> 31;
      const uint32_t c1 = h0, c2 = h0 + h1, c3 = c2 + h2, c4 = c3 + h3;
      const uint32_t s = quad * 4u;
      sts_u16(oa, s);
      sts_u16(oa + 64u * c1, s + 1u);
      sts_u16(oa + 64u * c2, s + 2u);
      sts_u16(oa + 64u * c3, s + 3u);
      oa += 64u * c4;
    };
    if (nsteps == (uint32_t)(kChunk / 4)) {
#pragma unroll
      for (int kk = 0; kk < kChunk / 4; ++kk) test_quad(quads[kk]);
    } else {
#pragma unroll
      for (int kk = 0; kk < kChunk / 4; ++kk) {
        if ((uint32_t)kk >= nsteps) break;
        test_quad(quads[kk]);
      }
    }
  }
  flush((oa - lbase) >> 6);
  __syncwarp();
  float fx = f3[0].x + f3[0].y, fy = f3[1].x + f3[1].y, fz = f3[2].x + f3[2].y;
#pragma unroll
  for (int o = 8; o < 32; o <<= 1) {
    fx += __shfl_xor_sync(0xffffffffu, fx, o);
    fy += __shfl_xor_sync(0xffffffffu, fy, o);
    fz += __shfl_xor_sync(0xffffffffu, fz, o);
  }
  if (valid && q == 0) {
    if (max3abs(fx, fy, fz) < kStage) {
      stage_add3(smem_u32(pl.A), 4u * pl.slots, hs, fx, fy, fz);
    } else {
      const uint32_t g = d.home_g0 + h;
      share_global(b, g, 0, fx, bad);
      share_global(b, g, 1, fy, bad);
      share_global(b, g, 2, fz, bad);
    }
  }
  if (ENERGY) {
    ce[0] = warp_sum((double)(en[0].x + en[0].y));
    ce[1] = warp_sum((double)(en[1].x + en[1].y));
    ce[2] = warp_sum((double)(en[2].x + en[2].y));
    ce[3] = (double)warp_sum(npair);
  }
}

// Global-memory path of an item whose stage does not fit: lanes are 32
// consecutive home atoms; the half-shell rule and the fixed-point sums are
// the same, with the shares added straight to the global sums.
template <int NT, bool ENERGY>
__device__ void consume_task_global3(const ForceBufs &b, const ItemDesc3<NT> &d, uint32_t t,
                                     double (&ce)[4], bool &bad) {
  const int lane = threadIdx.x & 31;
  const int nseg = d.nseg, z0 = d.z0, nz = d.nz;
  const uint32_t hbeg = d.off[0][1];
  const uint32_t H = d.H;
  double s[4] = {0.0, 0.0, 0.0, 0.0};
  for (uint32_t gi = t; gi * 32 < H; gi += d.ntask) {
    const uint32_t h = gi * 32 + lane;
    const bool valid = h < H;
    const uint32_t hh = valid ? h : H - 1;
    int lo = 1, hi = nseg;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (d.off[0][mid] - hbeg <= hh) lo = mid; else hi = mid - 1;
    }
    const int kmin = __reduce_min_sync(0xffffffffu, lo);
    const int kmax = __reduce_max_sync(0xffffffffu, lo);
    const uint32_t gh = d.home_g0 + hh;
    const float4 p = b.rs[gh];
    const float xi = p.x - d.sx[0], yi = p.y - d.sy[0], zi = p.z - d.sz_mid;
    const int ti = NT == 1 ? 0 : __float_as_int(p.w);
    float fx = 0.f, fy = 0.f, fz = 0.f, pe = 0.f, pes = 0.f, vir = 0.f;
    uint32_t np = 0;
    for (int c = 0; c < kCols; ++c) {
      for (int k = kmin - 1; k <= kmax + 1; ++k) {
        // home column: cell z0 - 1 lies wholly before the home atoms
        if (c == 0 && k == 0) continue;
        const int zc = (z0 - 1 + k + nz) % nz;
        const uint32_t key = d.kbase[c] + (uint32_t)zc;
        const float sz = k == 0 ? d.sz_lo : (k == nseg + 1 ? d.sz_hi : d.sz_mid);
        const bool later_only = c == 0 && k <= nseg;  // home cells: partners after gh
        for (uint32_t j = b.start[key]; j < b.start[key + 1]; ++j) {
          const float4 qj = b.rs[j];
          const float dx = xi - (qj.x - d.sx[c]), dy = yi - (qj.y - d.sy[c]),
                      dz = zi - (qj.z - sz);
          const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
          const int kk = NT == 1 ? 0 : ti * NT + __float_as_int(qj.w);
          if (!valid || !(r2 < d.lj.rc2[kk]) || !(r2 > 0.0f) || (later_only && j <= gh)) continue;
          const float inv = rcp_approx(r2);
          const float sr2 = d.lj.s2[kk] * inv;
          const float sr6 = sr2 * sr2 * sr2;
          const float f = d.lj.e24[kk] * sr6 * fmaf(2.0f, sr6, -1.0f) * inv;
          const float ax = f * dx, ay = f * dy, az = f * dz;
          fx += ax;
          fy += ay;
          fz += az;
          share_global(b, j, 0, -ax, bad);
          share_global(b, j, 1, -ay, bad);
          share_global(b, j, 2, -az, bad);
          if (ENERGY) {
            const float u = d.lj.e4[kk] * sr6 * (sr6 - 1.0f);
            pe += u;
            pes += u - d.lj.ush[kk];
            vir += f * r2;
            np += 2u;
          }
        }
      }
    }
    if (valid) {
      share_global(b, gh, 0, fx, bad);
      share_global(b, gh, 1, fy, bad);
      share_global(b, gh, 2, fz, bad);
    }
    if (ENERGY) {
      s[0] += warp_sum((double)pe);
      s[1] += warp_sum((double)pes);
      s[2] += warp_sum((double)vir);
      s[3] += (double)warp_sum(np);
    }
  }
  for (int k = 0; k < 4; ++k) ce[k] = s[k];
}

// ---- the kernel ---------------------------------------------------------------

template <int NT, bool ENERGY, int kProd, int kCons>
__global__ void __launch_bounds__((kProd + kCons) * 32, 2) k_force_half(ForceBufs b) {
  pdl_enter();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ ItemDesc3<NT> desc[2];
  __shared__ Scratch3 sc;
  __shared__ uint64_t full[2], empty[2], landed[2];
  __shared__ double cle[2][kWinCap][4];
  __shared__ int abort_flag, wait_ok;
  __shared__ uint32_t next_item;

  const uint32_t slots = padded_slots3((uint32_t)b.cap_half);
  const uint32_t sbytes = stage_bytes3(slots, NT), wbytes = warp_bytes3(slots);
  const uint32_t pbytes = plane_bytes3(slots, NT);
  auto stage = [&](int k) {
    unsigned char *base = smem_raw + (size_t)k * sbytes;
    float *f = reinterpret_cast<float *>(base);
    Stage p;
    p.X = f;
    p.Y = f + slots;
    p.Z = f + 2 * slots;
    p.T = NT > 1 ? reinterpret_cast<uint32_t *>(f + 3 * slots) : nullptr;
    p.A = reinterpret_cast<uint32_t *>(base + pbytes);
    p.slots = slots;
    return p;
  };
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t polls = b.wait_polls ? b.wait_polls : kWaitPolls;
  // the accumulators start cleared; retire_item3 clears them after each use
  for (uint32_t i = threadIdx.x; i < 2u * 6u * slots; i += blockDim.x) {
    const int k = i / (6u * slots);
    stage(k).A[i - k * 6u * slots] = 0u;
  }
  if (threadIdx.x == 0) {
    for (int k = 0; k < 2; ++k) {
      mbar_init(&full[k], 1);
      mbar_init(&empty[k], kCons);
      mbar_init(&landed[k], 1);
    }
    abort_flag = 0;
    mbar_fence_init();
  }
  __syncthreads();
  const volatile int *abort_v = &abort_flag;

  if (warp < kProd) {
    auto wait_empty = [&](int bf, uint32_t parity) -> bool {
      if (threadIdx.x == 0) {
        const bool ok = mbar_wait_or_abort(&empty[bf], parity, &kNeverAbort, polls);
        wait_ok = ok;
        if (!ok) {
          atomicOr(&b.status[desc[bf].sys], kStatusWaitTimeout);
          abort_flag = 1;
        }
      }
      producer_sync<kProd>();
      const bool ok = wait_ok;
      producer_sync<kProd>();
      return ok;
    };
    auto done_claiming = [&]() {
      if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(b.queue + 1, 1u) == gridDim.x - 1) {
          atomicExch(b.queue, 0u);
          atomicExch(b.queue + 1, 0u);
        }
      }
    };
    uint32_t lphase0 = 0u, lphase1 = 0u, running = 0;
    uint32_t n = 0;
    for (;; ++n) {
      if (threadIdx.x == 0) next_item = atomicAdd(b.queue, 1u);
      const int bf = n & 1;
      if (n >= 2) {
        if (!wait_empty(bf, ((n >> 1) - 1) & 1u)) {
          done_claiming();
          return;
        }
        retire_item3<NT, kProd, ENERGY>(b, desc[bf], stage(bf), cle[bf]);
      }
      producer_sync<kProd>();
      const uint32_t item = next_item;
      producer_sync<kProd>();
      if (item >= b.nitems) {
        done_claiming();
        if (threadIdx.x == 0) {
          desc[bf].item = kNone;
          mbar_arrive(&full[bf]);
        }
        break;
      }
      const bool ok = produce_item3<NT, kProd>(b, item, desc[bf], sc, stage(bf), &landed[bf],
                                               bf ? lphase1 : lphase0, running, kCons);
      if (!ok) {
        done_claiming();
        if (threadIdx.x == 0) abort_flag = 1;
        return;
      }
      // test hook (PB test entry only): withhold the first hand-off so that
      // the consumers' bounded wait runs out
      const bool withhold = (b.test_flags & 1u) && n == 0;
      if (threadIdx.x == 0 && !withhold) mbar_arrive(&full[bf]);
    }
    if (n >= 1) {
      const uint32_t m = n - 1;
      const int bf = m & 1;
      if (!wait_empty(bf, (m >> 1) & 1u)) return;
      retire_item3<NT, kProd, ENERGY>(b, desc[bf], stage(bf), cle[bf]);
    }
    return;
  }

  // consumers
  const int cw = warp - kProd;
  uint16_t *mylist =
      reinterpret_cast<uint16_t *>(smem_raw + 2 * (size_t)sbytes + (size_t)cw * wbytes);
  uint16_t *tb = mylist + 32 * kListLen;
  bool bad = false;
  for (uint32_t n = 0;; ++n) {
    const int bf = n & 1;
    bool ok = lane != 0 || mbar_wait_or_abort(&full[bf], (n >> 1) & 1u, abort_v, polls);
    ok = __shfl_sync(0xffffffffu, ok, 0);
    if (!ok) {
      if (lane == 0 && !*abort_v) atomicOr(&b.status[0], kStatusWaitTimeout);
      return;
    }
    const ItemDesc3<NT> &d = desc[bf];
    if (d.item == kNone) break;
    const Stage pbuf = stage(bf);
    if (!d.skip) {
      if (!d.overflow) {
        const uint32_t first = ((uint32_t)cw + (uint32_t)kCons - d.base) % (uint32_t)kCons;
        for (uint32_t cl = first; cl < d.nclus; cl += kCons) {
          double ce[4];
          consume_cluster3<NT, ENERGY>(b, d, pbuf, cl, mylist, tb, ce, bad);
          if (ENERGY && lane == 0)
            for (int k = 0; k < 4; ++k) cle[bf][cl][k] = ce[k];
        }
      } else {
        for (uint32_t t = (uint32_t)cw; t < d.ntask; t += kCons) {
          double ce[4];
          consume_task_global3<NT, ENERGY>(b, d, t, ce, bad);
          if (ENERGY && lane == 0)
            for (int k = 0; k < 4; ++k) cle[bf][t][k] = ce[k];
        }
      }
      if (__any_sync(0xffffffffu, bad)) {
        if (lane == 0) atomicOr(&b.status[d.sys], kStatusNonFinite);
        bad = false;
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[bf]);
  }
}

// Fixed-point sums -> FP32 forces in particle order, and the sums cleared.
// One block per integration block of the system map (sorted slots of a
// system are the same range as its atoms).
__global__ void __launch_bounds__(256) k_force_finish(ForceBufs b) {
  pdl_enter();
  const BlockMap m = b.map[blockIdx.x];
  if (b.steps_left != nullptr && b.steps_left[m.sys] == 0) return;
  const size_t n3 = b.nacc;
  for (uint32_t t = threadIdx.x; t < m.n; t += blockDim.x) {
    const uint32_t s = m.i0 + t;
    float f[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const long long fine = (long long)b.facc[c * n3 + s];
      const long long coarse = (long long)b.fbig[c * n3 + s];
      b.facc[c * n3 + s] = 0ull;
      if (coarse != 0) b.fbig[c * n3 + s] = 0ull;
      f[c] = (float)((double)fine * (1.0 / 4294967296.0) + (double)coarse * 0.5);
    }
    b.F[b.pid[s]] = make_float4(f[0], f[1], f[2], 0.0f);
  }
}

template <typename K>
int resident_ctas3(K kern, int threads, size_t smem) {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, threads, smem) != cudaSuccess) n = 1;
  return n > 0 ? n : 1;
}

int sm_count3() {
  static int n = 0;
  if (n == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 1;
  }
  return n;
}

constexpr int kProd3 = 4, kCons3 = 8;

template <int NT, bool E>
cudaError_t launch_half_nt(const ForceBufs &b, cudaStream_t s) {
  const size_t smem = smem_bytes3((uint32_t)b.cap_half, kCons3, NT);
  auto kern = k_force_half<NT, E, kProd3, kCons3>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const long slots = (long)resident_ctas3(kern, (kProd3 + kCons3) * 32, smem) * sm_count3();
  const unsigned grid = (unsigned)std::min<long>(slots, (long)b.nitems);
  e = launch_pdl(kern, dim3(grid), dim3((kProd3 + kCons3) * 32), smem, s, b);
  if (e != cudaSuccess) return e;
  return launch_pdl(k_force_finish, dim3(b.nblocks), dim3(256), 0, s, b);
}

template <bool E>
cudaError_t launch_half_e(const ForceBufs &b, int nt_max, cudaStream_t s) {
  switch (nt_max) {
    case 1: return launch_half_nt<1, E>(b, s);
    case 2: return launch_half_nt<2, E>(b, s);
    case 3: case 4: return launch_half_nt<4, E>(b, s);
    default: return launch_half_nt<8, E>(b, s);
  }
}

}  // namespace

int force_half_max_capacity(int nt) {
  uint32_t cap = 64;
  while (smem_bytes3(cap + 64, kCons3, nt) <= 180u * 1024u) cap += 64;
  return (int)cap;
}

int force_half_smem_per_cta(int cap, int nt) {
  return (int)smem_bytes3((uint32_t)cap, kCons3, nt) + 15 * 1024;
}

cudaError_t launch_force_half(const ForceBufs &b, int nt_max, bool energy, cudaStream_t s) {
  if (b.nitems == 0) return cudaSuccess;
  return energy ? launch_half_e<true>(b, nt_max, s) : launch_half_e<false>(b, nt_max, s);
}

}  // namespace pb
