// Lennard-Jones pair forces over the cell list.
//
// Replaces cudaParticleMD::calcForce (cudaParticleMD.cu:24-69):
// calcF_IJpairWithBlock_F4<MDpairForce<potentialLJ>> on a (cells x 27) grid
// writing 27 partial-force planes tmp81N, followed by reduce27_F4
// (kerneltemplate.hh:229-294, kerneltemplate.hh:523-565, kernelinline.hh:86-96,
// kernelfuncs.cu:935-949).  The physics is the reference's: truncated,
// unshifted LJ, F_i = sum_{j != i, r < rc} 24 eps (s/r)^6 (2 (s/r)^6 - 1) / r^2
// (r_i - r_j) with the minimum image, over the 27-cell stencil.  No 81 N
// scratch: each atom's force is summed in registers and written once.
//
// Work items.  One work item = (system, x-y column of cells, run of z cells
// [z0, z1)); its stage is the 3 x 3 neighbour columns over z cells
// [z0 - 1, z1] (periodic halo cells included).
//
// Persistent, warp-specialised CTAs.  Each CTA walks the items blockIdx.x,
// blockIdx.x + gridDim.x, ... with two stage buffers.  Warp 0 is the
// producer: for item n + 1 it reads the cell starts, lands the stage in the
// free buffer with 1-D bulk copies (cp.async.bulk, mbarrier completion, no
// multicast) from the structure-of-arrays mirrors of the sorted positions,
// applies the frame shifts, and searches the z window of every (cluster,
// column).  The other warps are consumers: they compute item n from the other
// buffer meanwhile, and move on to item n + 1 as soon as the producer
// publishes it.  mbarriers hand buffers back and forth (full: producer to
// consumers; empty: consumers to producer); every wait is bounded.
//
// Stage layout.  Each staged column is a run of whole 4-atom quads: the bulk
// copies move 16-byte aligned runs of the x, y, z (and type) mirrors, so up to
// 3 atoms of the neighbouring cells ride along at each end of a run; the
// producer turns those into far atoms (x, y = 1e30) whose z keeps the column
// sorted.  Mirror runs start at the same offset modulo 4 whether a system runs
// alone or in a batch, so the layout, and every sum, is the same in both.
//
// Coordinate frame.  Positions are absolute FP32 coordinates.  Each item moves
// all staged atoms into one frame by subtracting 0 or L per axis: a neighbour
// image below the box (atoms near the top face) and, in items on the top face,
// every non-wrapped atom, get x - L.  The subtraction only ever applies to
// coordinates >= L/2, where it is exact (Sterbenz), so displacements x_i - x_j
// in the frame are the minimum-image displacements with no rounding beyond
// the subtraction itself, even in a 190-sigma box.  Work items are laid out
// so that a top-face item's cells all lie above the box middle.
//
// Compute.  Cells are sorted by z and atoms within a cell by z, so every
// staged column is one z-sorted array.  A consumer warp takes a cluster of 8
// consecutive home atoms (lane & 7) and splits the candidates 4 ways
// (lane >> 3).  It writes the quads of the cluster's 9 column windows into one
// flat table (padded to whole chunks with a quad of far atoms), so the
// candidate loop runs over one sequence with no per-column tails.  Then
//   phase 1  tests 4 candidates per step (one quad, packed FP32x2 arithmetic)
//            against rc^2 (1 + 2^-10) and appends the hits to a per-lane index
//            list in shared memory (no divergent force code);
//   phase 2  recomputes each listed pair exactly, applies the exact cutoff
//            r^2 < rc^2 of the pair's types (which also drops the self pair,
//            r^2 = 0), and evaluates the force, two list entries per step in
//            packed FP32x2 arithmetic.
// The 4 partial sums of an atom are combined with two warp shuffles.
// Clusters go to consumers round-robin over the CTA's whole item sequence;
// a cluster's arithmetic does not depend on which warp runs it, and energy
// sums are kept per cluster and added in cluster order.  An item whose stage
// exceeds the shared-memory capacity computes from global memory instead
// (slower, same result) and raises a status bit.
#include <algorithm>
#include <type_traits>

#include "force_common.cuh"

namespace pb {
namespace {

// One work item as the consumers see it (written by the producer).
template <int NT>
struct ItemDesc {
  // index within column c of the first staged atom of z cell k (k = 0 is image
  // cell z0 - 1, k = nseg + 1 is image cell z1); entry nseg + 2 is the column's count
  uint32_t off[9][kMaxSeg + 3];
  uint32_t ps[10];     // first slot of each column's region; ps[9] = end
  uint32_t kbase[9];   // packed key of z cell 0 of each column
  float sx[9], sy[9];  // frame shift of each column (0 or L)
  float sz_lo, sz_mid, sz_hi;  // frame shift of staged cell 0, 1..nseg, nseg + 1
  uint32_t item, sys, home_g0, hb, H, nclus, ntask, sentinel, base;
  int z0, nz, nseg;
  int periodic;        // 0: open box (neighbour columns may be absent, no z images)
  int skip;            // the system's step budget is spent
  int overflow;        // the stage exceeds the capacity: global-memory path
  LJLocal<NT> lj;
  // z window of each (cluster, column): first quad, quads, flat offset; per
  // cluster the total and the longest (at least 2)
  uint16_t q0[kWinCap][9], len[kWinCap][9], pre[kWinCap][9];
  uint16_t Q[kWinCap], M[kWinCap];
};

// Producer scratch: global cell starts and counts of the item being staged,
// and its copy runs (piece p of column c at index 3 c + p).
struct Scratch {
  uint32_t gstart[9][kMaxSeg + 3];
  uint32_t cnt[9][kMaxSeg + 3];
  uint32_t dst[27], lead[27], n[27], alen[27];
  uint32_t src[27];    // mirror slot of each run's first (16-byte aligned) slot
  float shift[27][3];  // frame shift of each run
};

// Slots of a stage buffer for `cap` staged atoms: each of up to 3 copy runs
// per column brings at most 6 neighbouring atoms, plus one quad of far atoms
// that pads the last chunk of every quad table.
__host__ __device__ __forceinline__ uint32_t padded_slots(uint32_t cap) {
  return ((cap + 162u + 3u) & ~3u) + 4u;
}

__host__ __device__ __forceinline__ uint32_t plane_bytes(uint32_t slots, int nt) {
  return (slots * (nt > 1 ? 16u : 12u) + 15u) & ~15u;
}

// Bytes of one consumer warp's pair lists plus its quad table.
__host__ __device__ __forceinline__ uint32_t warp_bytes(uint32_t slots) {
  return ((32u * kListLen * 2u + (slots / 4u + kChunk) * 2u) + 15u) & ~15u;
}

// Dynamic shared memory of one CTA: two stage buffers and the consumers' lists.
__host__ __device__ __forceinline__ uint32_t smem_bytes(uint32_t cap, int consumers, int nt) {
  const uint32_t slots = padded_slots(cap);
  return 2u * plane_bytes(slots, nt) + (uint32_t)consumers * warp_bytes(slots);
}

// MODE kModeCapped: relaxation force of the steepest-descent path, with the
// pair distance floored at sigma/2 so that overlapping random starts give
// finite forces.  MODE kModeSoftCore: the soft-core force of potentialSC
// (kernelinline.hh:136-158) as MDpairForce applies it (kerneltemplate.hh:530-564):
// f0 cos(r / rc * pi / 2) times the unit vector, zero beyond rc.
template <int NT, bool ENERGY, typename Acc, int MODE = kModeLJ>
struct PairAcc {
  Acc fx = 0, fy = 0, fz = 0, pe = 0, pes = 0, vir = 0;
  uint32_t n = 0;
  template <int M>
  __device__ __forceinline__ void add(const LJLocal<M> &lj, int k, float dx, float dy, float dz,
                                      float r2) {
    if (MODE == kModeSoftCore) {
      const float r = sqrtf(r2);
      if (r > lj.sc_rc) return;
      const float mag = lj.sc_f0 * (float)cos((double)(r / lj.sc_rc) * 3.14159265358979323846 / 2);
      const float f = mag * rsqrtf(r2);
      fx += (Acc)(f * dx);
      fy += (Acc)(f * dy);
      fz += (Acc)(f * dz);
      return;
    }
    if (MODE == kModeCapped) r2 = fmaxf(r2, 0.25f * lj.s2[k]);
    const float inv = rcp_approx(r2);
    const float sr2 = lj.s2[k] * inv;
    const float sr6 = sr2 * sr2 * sr2;
    const float f = lj.e24[k] * sr6 * fmaf(2.0f, sr6, -1.0f) * inv;
    fx += (Acc)(f * dx);
    fy += (Acc)(f * dy);
    fz += (Acc)(f * dz);
    if (ENERGY) {
      const float u = lj.e4[k] * sr6 * (sr6 - 1.0f);
      pe += (Acc)(0.5f * u);
      pes += (Acc)(0.5f * (u - lj.ush[k]));
      vir += (Acc)(0.5f * f * r2);
      ++n;
    }
  }
};

// Packed accumulators of the phase-2 fast path (FP32 sums, LJ or capped law):
// each lane keeps two partial sums per quantity, one per list-entry parity.
template <bool ENERGY>
struct PairAcc2 {
  float2 fx = {0.f, 0.f}, fy = {0.f, 0.f}, fz = {0.f, 0.f};
  float2 pe = {0.f, 0.f}, pes = {0.f, 0.f}, vir = {0.f, 0.f};
  uint32_t n = 0;
};

// Global-memory path (stage overflow): lanes are 32 consecutive home atoms,
// candidates of one z cell of one column, frame shifts applied per pair.
template <int NT, bool ENERGY, bool SELF, typename Acc, int MODE>
__device__ __forceinline__ void global_range(const float4 *__restrict__ P, uint32_t jb,
                                             uint32_t je, float xi, float yi, float zi, int ti,
                                             float sx, float sy, float sz, uint32_t self,
                                             const LJLocal<NT> &lj,
                                             PairAcc<NT, ENERGY, Acc, MODE> &a) {
  for (uint32_t j = jb; j < je; ++j) {
    const float4 q = P[j];
    const float dx = xi - (q.x - sx), dy = yi - (q.y - sy), dz = zi - (q.z - sz);
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    const int k = NT == 1 ? 0 : ti * NT + __float_as_int(q.w);
    if (r2 < lj.rc2[k] && (!SELF || j != self)) a.add(lj, k, dx, dy, dz, r2);
  }
}

// Phase 2, general form: one listed pair per step, any force law and any
// accumulator type.  Entries are padded slots; the exact cutoff drops the
// candidates phase 1 admitted through its margin and the self pair.
template <int NT, bool ENERGY, typename Acc, int MODE>
__device__ __forceinline__ void flush_scalar(const float *X, const float *Y, const float *Z,
                                             const uint32_t *T, const uint16_t *list,
                                             uint32_t cnt, int lane, float xi, float yi, float zi,
                                             int ti, const LJLocal<NT> &lj,
                                             PairAcc<NT, ENERGY, Acc, MODE> &a) {
  for (uint32_t k = 0; k < cnt; ++k) {
    const uint32_t j = list[k * 32 + lane];
    const float dx = xi - X[j], dy = yi - Y[j], dz = zi - Z[j];
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    const int kk = NT == 1 ? 0 : ti * NT + (int)T[j];
    if (r2 < lj.rc2[kk] && r2 > 0.0f) a.add(lj, kk, dx, dy, dz, r2);
  }
}

// Phase 2, fast form (FP32 sums, LJ or capped law): two list entries per step
// in packed FP32x2 arithmetic; the force of an entry outside the exact cutoff
// (or past the lane's count) is selected to zero.
template <int NT, bool ENERGY, int MODE>
__device__ __forceinline__ void flush_packed(const float *X, const float *Y, const float *Z,
                                             const uint32_t *T, const uint16_t *list,
                                             uint32_t cnt, int lane, float xi, float yi, float zi,
                                             int ti, const LJLocal<NT> &lj,
                                             PairAcc2<ENERGY> &a) {
  const float2 m1 = make_float2(-1.0f, -1.0f);
  const float2 xi2 = make_float2(xi, xi), yi2 = make_float2(yi, yi), zi2 = make_float2(zi, zi);
  const float2 two = make_float2(2.0f, 2.0f), mone = make_float2(-1.0f, -1.0f);
  const float2 half = make_float2(0.5f, 0.5f);
  float2 s2 = make_float2(lj.s2[0], lj.s2[0]), e24 = make_float2(lj.e24[0], lj.e24[0]);
  float2 e4 = make_float2(lj.e4[0], lj.e4[0]), ush = make_float2(lj.ush[0], lj.ush[0]);
  float rc2a = lj.rc2[0], rc2b = lj.rc2[0];
  // shared-memory byte addresses of the planes and of this lane's entries
  const uint32_t xa = smem_u32(X), ya = smem_u32(Y), za = smem_u32(Z);
  const uint32_t la = smem_u32(list) + 2u * (uint32_t)lane;
  for (uint32_t k = 0; k < cnt; k += 2) {
    const uint32_t j0 = lds_u16(la + 64u * k);
    const uint32_t j1 = lds_u16(la + 64u * min(k + 1, cnt - 1));
    const bool v1 = k + 1 < cnt;
    if (NT > 1) {
      const int ka = ti * NT + (int)T[j0], kb = ti * NT + (int)T[j1];
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
    const bool ina = r2.x < rc2a && r2.x > 0.0f;
    const bool inb = v1 && r2.y < rc2b && r2.y > 0.0f;
    float2 r2c = r2;
    if (MODE == kModeCapped) {
      const float2 fl = __fmul2_rn(make_float2(0.25f, 0.25f), s2);
      r2c = make_float2(fmaxf(r2.x, fl.x), fmaxf(r2.y, fl.y));
    }
    const float2 inv = make_float2(rcp_approx(r2c.x), rcp_approx(r2c.y));
    const float2 sr2 = __fmul2_rn(s2, inv);
    const float2 sr6 = __fmul2_rn(__fmul2_rn(sr2, sr2), sr2);
    const float2 t = __ffma2_rn(two, sr6, mone);
    float2 f = __fmul2_rn(__fmul2_rn(__fmul2_rn(e24, sr6), t), inv);
    f.x = ina ? f.x : 0.0f;
    f.y = inb ? f.y : 0.0f;
    a.fx = __ffma2_rn(f, dx, a.fx);
    a.fy = __ffma2_rn(f, dy, a.fy);
    a.fz = __ffma2_rn(f, dz, a.fz);
    if (ENERGY) {
      float2 u = __fmul2_rn(__fmul2_rn(e4, sr6), __fadd2_rn(sr6, mone));
      u.x = ina ? u.x : 0.0f;
      u.y = inb ? u.y : 0.0f;
      float2 us = __fadd2_rn(u, make_float2(-ush.x, -ush.y));
      us.x = ina ? us.x : 0.0f;
      us.y = inb ? us.y : 0.0f;
      a.pe = __ffma2_rn(half, u, a.pe);
      a.pes = __ffma2_rn(half, us, a.pes);
      a.vir = __ffma2_rn(__fmul2_rn(half, f), r2c, a.vir);
      a.n += (uint32_t)ina + (uint32_t)inb;
    }
  }
}

// ---- producer ---------------------------------------------------------------

// Set up item `item` in descriptor `d` and stage buffer `pl` (the kProd
// producer warps together).  Returns false when the wait for the bulk copies
// gave up.
template <int NT, int MODE, int kProd, int kCons>
__device__ bool produce_item(const ForceBufs &b, uint32_t item, ItemDesc<NT> &d, Scratch &sc,
                             const Planes &pl, uint32_t &running) {
  constexpr int kPT = kProd * 32;  // producer threads
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
  if (skip) {  // a system whose step budget is spent keeps its state
    producer_sync<kProd>();
    return true;
  }
  const SysDesc &S = b.sys[it.sys];
  const Grid g = S.g;
  const uint32_t mirror0 = S.mirror0, atom0 = S.atom0, scap = S.cap;
  const int nx = g.n[0], ny = g.n[1], nz = g.n[2];
  const int z0 = it.z0, z1 = it.z1, nseg = z1 - z0;
  const int ncell = nseg + 2;  // staged cells per column
  const bool per = g.periodic != 0;
  for (int t = pt; t < NT * NT; t += kPT) {
    const LJTable &Tb = b.lj[S.lj];
    const int a = t / NT, c = t % NT;
    const int k = a * Tb.nt + c;
    d.lj.s2[t] = Tb.s2[k];
    d.lj.e24[t] = Tb.e24[k];
    d.lj.e4[t] = Tb.e4[k];
    d.lj.rc2[t] = MODE == kModeSoftCore ? fminf(Tb.rc2[k], b.sc_rc * b.sc_rc) : Tb.rc2[k];
    d.lj.ush[t] = Tb.ushift[k];
  }
  if (pt < 9) {
    const int cx = it.cx, cy = it.cy;
    const int c = pt;
    const int ax = cx + c / 3 - 1, ay = cy + c % 3 - 1;
    const int wx = ax < 0 ? -1 : (ax >= nx ? 1 : 0);
    const int wy = ay < 0 ? -1 : (ay >= ny ? 1 : 0);
    // frame: F = L on the top face; staged = x + w L - F, so the shift is F - w L
    // (an open box has no images and no frame shift)
    const float Fx = per && cx == nx - 1 ? g.L[0] : 0.0f, Fy = per && cy == ny - 1 ? g.L[1] : 0.0f;
    d.sx[c] = per ? Fx - (float)wx * g.L[0] : 0.0f;
    d.sy[c] = per ? Fy - (float)wy * g.L[1] : 0.0f;
    d.kbase[c] = it.kbase[c];
  }
  // an item on the top face works in the frame shifted down by L, where the
  // shifts of its atoms (all in the upper half) are exact; a whole column
  // keeps the unshifted frame and rounds only the image above its top
  const float Fz = per && z1 == nz && z0 > 0 ? g.L[2] : 0.0f;
  const float sz_lo = per && z0 == 0 ? Fz + g.L[2] : Fz;  // image z0 - 1 wraps below when z0 == 0
  const float sz_hi = per && z1 == nz ? Fz - g.L[2] : Fz;  // image z1 wraps above when z1 == nz
  if (pt == 0) {
    d.sz_lo = sz_lo;
    d.sz_mid = Fz;
    d.sz_hi = sz_hi;
    d.z0 = z0;
    d.nz = nz;
    d.nseg = nseg;
    d.periodic = per;
    d.lj.sc_rc = b.sc_rc;
    d.lj.sc_f0 = b.sc_f0;
  }
  // cell starts and counts of the 9 x ncell staged cells; in an open box a
  // column past a face, or a cell past the bottom or top, is empty
  for (int t = pt; t < 9 * ncell; t += kPT) {
    const int c = t / ncell, k = t % ncell;
    const int zr = z0 - 1 + k, zc = (zr + nz) % nz;
    uint32_t s0 = 0, s1 = 0;
    if (per || (it.kbase[c] != kNoCell && zr >= 0 && zr < nz)) {
      const uint32_t key = it.kbase[c] + (uint32_t)zc;
      s0 = b.start[key];
      s1 = b.start[key + 1];
    }
    sc.gstart[c][k] = s0;
    sc.cnt[c][k] = s1 - s0;
  }
  producer_sync<kProd>();
  // exclusive prefix over the cells of each column, one warp per column
  for (int c = pw; c < 9; c += kProd) {
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
  // copy runs: piece 0 = image cell z0 - 1 when z0 == 0, piece 2 = image cell
  // z1 when z1 == nz, piece 1 = the cells between (consecutive z, one run)
  const int a_end = z0 == 0 ? 1 : 0, c_beg = z1 == nz ? ncell - 1 : ncell;
  const uint32_t H = d.off[4][nseg + 1] - d.off[4][1];
  const uint32_t nclus = (H + 7) / 8;
  if (pw == 0) {
    uint32_t n = 0, m0 = 0, ma = 0, alen = 0;
    if (lane < 27) {
      const int c = lane / 3, p = lane % 3;
      const int k0 = p == 0 ? 0 : (p == 1 ? a_end : c_beg);
      const int k1 = p == 0 ? a_end : (p == 1 ? c_beg : ncell);
      n = d.off[c][k1] - d.off[c][k0];
      if (n > 0) {
        m0 = mirror0 + (sc.gstart[c][k0] - atom0);
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
    // frame shift of each run: the column's x, y shift and the run's z shift
    float rx = 0.f, ry = 0.f, rz = 0.f;
    if (lane < 27) {
      const int c = lane / 3, pp = lane % 3;
      rx = d.sx[c];
      ry = d.sy[c];
      rz = pp == 0 ? sz_lo : (pp == 1 ? Fz : sz_hi);
      sc.dst[lane] = dst;
      sc.src[lane] = ma;
      sc.lead[lane] = m0 - ma;
      sc.n[lane] = n;
      sc.alen[lane] = alen;
      sc.shift[lane][0] = rx;
      sc.shift[lane][1] = ry;
      sc.shift[lane][2] = rz;
      if (lane % 3 == 0) d.ps[lane / 3] = dst;
    }
    // the system's own capacity decides: the same path alone or batched
    const bool overflow = total + 4u > padded_slots(scap) || nclus > (uint32_t)kWinCap;
    if (lane == 0) {
      d.ps[9] = total;
      d.H = H;
      d.home_g0 = sc.gstart[4][1];
      d.overflow = overflow;
      if (overflow) {
        d.ntask = min((H + 31) / 32, (uint32_t)kWinCap);
        atomicOr(&b.status[it.sys], kStatusSmemOverflow);
      }
    }
  }
  producer_sync<kProd>();
  if (d.overflow) return true;
  const uint32_t total = d.ps[9];
  if (total > 0) {
    // the runs' 16-byte quads, all producer threads, each run moved into the
    // item's frame on the way (x - 0 is x, so unshifted runs pass unchanged);
    // kCopyBatch quads per thread are loaded before any is stored
    constexpr int kB = NT > 1 ? kCopyBatch / 2 : kCopyBatch;  // the type plane takes registers
    const uint32_t nq = total >> 2;
    int p = 0;
    for (uint32_t u0 = pt; u0 < nq; u0 += kB * kPT) {
      float4 vx[kB], vy[kB], vz[kB];
      uint4 vt[NT > 1 ? kB : 1];
      int pr[kB];
#pragma unroll
      for (int k = 0; k < kB; ++k) {
        const uint32_t u = u0 + (uint32_t)k * kPT;
        pr[k] = -1;
        if (u < nq) {
          while (4u * u >= sc.dst[p] + sc.alen[p]) ++p;  // runs in slot order
          pr[k] = p;
          const uint32_t g = sc.src[p] + (4u * u - sc.dst[p]);
          vx[k] = ldg_f4(b.xs + g);
          vy[k] = ldg_f4(b.ys + g);
          vz[k] = ldg_f4(b.zs + g);
          if (NT > 1) vt[k] = ldg_u4(b.ts + g);
        }
      }
#pragma unroll
      for (int k = 0; k < kB; ++k) {
        if (pr[k] < 0) break;
        const uint32_t s = 4u * (u0 + (uint32_t)k * kPT);
        const float sx = sc.shift[pr[k]][0], sy = sc.shift[pr[k]][1], sz = sc.shift[pr[k]][2];
        sts_f4(smem_u32(pl.X + s), make_float4(vx[k].x - sx, vx[k].y - sx, vx[k].z - sx, vx[k].w - sx));
        sts_f4(smem_u32(pl.Y + s), make_float4(vy[k].x - sy, vy[k].y - sy, vy[k].z - sy, vy[k].w - sy));
        sts_f4(smem_u32(pl.Z + s), make_float4(vz[k].x - sz, vz[k].y - sz, vz[k].z - sz, vz[k].w - sz));
        if (NT > 1) *reinterpret_cast<uint4 *>(pl.T + s) = vt[k];
      }
    }
    producer_sync<kProd>();
    // neighbouring atoms that rode along become far atoms that keep z sorted
    if (pt < 27 && sc.alen[pt] > 0) {
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
    // the quad of far atoms that pads the last chunk of a table
    const uint32_t s = total + (uint32_t)(pt - 32 * (kProd - 1));
    pl.X[s] = kFar;
    pl.Y[s] = kFar;
    pl.Z[s] = kFar;
    if (NT > 1) pl.T[s] = 0u;
  }
  producer_sync<kProd>();
  // z windows of every (cluster, column)
  const int hp = 4 * 3 + 1;  // the home column's middle run holds home cells 1..nseg
  const uint32_t hb = sc.dst[hp] + sc.lead[hp] + (d.off[4][1] - d.off[4][a_end]);
  float rcmax2 = 0.f;
  for (int k = 0; k < NT * NT; ++k) rcmax2 = fmaxf(rcmax2, d.lj.rc2[k]);
  const float rcw = sqrtf(rcmax2) * 1.00001f + 1e-5f;
  for (uint32_t t = pt; t < 9u * nclus; t += kPT) {
    const uint32_t k = t / 9u, c = t - 9u * k;
    const float zmin = pl.Z[hb + k * 8];
    const float zmax = pl.Z[hb + min(k * 8 + 7, H - 1)];
    const uint32_t lo = d.ps[c], hi = d.ps[c + 1];
    const uint32_t a = lower_bound_z(pl.Z, lo, hi, zmin - rcw) >> 2;
    const uint32_t e = (upper_bound_z(pl.Z, lo, hi, zmax + rcw) + 3u) >> 2;
    d.q0[k][c] = (uint16_t)a;
    // empty unless ordered (an unsorted column, e.g. NaN positions, can
    // invert the two searches)
    d.len[k][c] = (uint16_t)(e > a ? e - a : 0u);
  }
  producer_sync<kProd>();
  for (uint32_t k = pt; k < nclus; k += kPT) {
    uint32_t s = 0, m = 2;
    for (int c = 0; c < 9; ++c) {
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

// Energy partials of a finished item: its per-cluster (or per-task) sums in
// cluster order.
template <int NT>
__device__ void write_partials(const ForceBufs &b, const ItemDesc<NT> &d, const double (*e)[4]) {
  double v[4] = {0.0, 0.0, 0.0, 0.0};
  if (!d.skip) {
    const uint32_t n = d.overflow ? d.ntask : d.nclus;
    for (uint32_t k = 0; k < n; ++k) {
      v[0] += e[k][0];
      v[1] += e[k][1];
      v[2] += e[k][2];
      v[3] += e[k][3];
    }
  }
  for (int k = 0; k < 4; ++k) b.partials[(size_t)d.item * 4 + k] = v[k];
}

// ---- consumers --------------------------------------------------------------

// One cluster of 8 home atoms (consumer warp, all 32 lanes); returns the
// cluster's energy sums in lane 0 (pe, shifted pe, virial, pairs).
template <int NT, bool ENERGY, typename Acc, int MODE>
__device__ __forceinline__ void consume_cluster(const ForceBufs &b, const ItemDesc<NT> &d,
                                                const Planes &pl, uint32_t cl, uint16_t *mylist,
                                                uint16_t *tb, double (&ce)[4]) {
  constexpr bool kPacked = std::is_same<Acc, float>::value && MODE != kModeSoftCore;
  const int lane = threadIdx.x & 31;
  const int il = lane & 7, q = lane >> 3;
  const float *X = pl.X, *Y = pl.Y, *Z = pl.Z;
  const uint32_t *T = pl.T;
  const uint32_t H = d.H, hb = d.hb;
  const uint32_t h = cl * 8 + il;
  const bool valid = h < H;
  const uint32_t hs = hb + (valid ? h : H - 1);
  const float xi = valid ? X[hs] : kNoAtom;
  const float yi = valid ? Y[hs] : kNoAtom;
  const float zi = valid ? Z[hs] : kNoAtom;
  // the particle index of the force store, fetched now so that its latency
  // passes during the pair loops
  const uint32_t pi = valid && q == 0 ? __ldg(b.pid + d.home_g0 + h) : 0u;
  const int ti = NT == 1 ? 0 : (int)T[hs];
  // the warp's quad table: lanes cover (column, index) pairs, column = idx / M
  // by a multiply-high (exact while 9 M^2 < 2^32)
  const uint32_t Q = d.Q[cl], M = d.M[cl];
  const uint32_t magic = 0xffffffffu / M + 1u;
  for (uint32_t idx = lane; idx < 9u * M; idx += 32) {
    const uint32_t c = __umulhi(idx, magic), i = idx - c * M;
    if (i < d.len[cl][c]) tb[table_pos(d.pre[cl][c] + i)] = (uint16_t)(d.q0[cl][c] + i);
  }
  for (uint32_t u = Q + lane; u < ((Q + 15u) & ~15u); u += 32)
    tb[table_pos(u)] = (uint16_t)d.sentinel;
  __syncwarp();

  float rcmax2 = 0.f;
  for (int k = 0; k < NT * NT; ++k) rcmax2 = fmaxf(rcmax2, d.lj.rc2[k]);
  // phase-1 bound with a margin: a superset of the exact test of phase 2
  const float2 nrc = make_float2(-rcmax2 * (1.0f + 1.0f / 1024.0f),
                                 -rcmax2 * (1.0f + 1.0f / 1024.0f));
  const float2 m1 = make_float2(-1.0f, -1.0f);
  PairAcc<NT, ENERGY, Acc, MODE> acc;
  PairAcc2<ENERGY> acc2;
  auto flush = [&](uint32_t cnt) {
    if constexpr (kPacked) {
      flush_packed<NT, ENERGY, MODE>(X, Y, Z, T, mylist, cnt, lane, xi, yi, zi, ti, d.lj, acc2);
    } else {
      flush_scalar<NT, ENERGY, Acc, MODE>(X, Y, Z, T, mylist, cnt, lane, xi, yi, zi, ti, d.lj,
                                          acc);
    }
  };
  const float2 xi2 = make_float2(xi, xi), yi2 = make_float2(yi, yi), zi2 = make_float2(zi, zi);
  // shared-memory byte addresses: candidate planes, and this lane's list
  // entries at lbase + 64 k (entry k of lane `lane`)
  const uint32_t xa = smem_u32(X), ya = smem_u32(Y), za = smem_u32(Z);
  const uint32_t lbase = smem_u32(mylist) + 2u * (uint32_t)lane;
  uint32_t oa = lbase;  // shared-memory address of this lane's next list entry
  // lane q tests quads u = q, q + 4, ... of the flat sequence, 4 per chunk; the
  // table pads the last chunk with the quad of far atoms
  for (uint32_t u0 = 0; u0 < Q; u0 += kChunk) {
    const uint32_t cnt = (oa - lbase) >> 6;
    if (__reduce_max_sync(0xffffffffu, cnt) > (uint32_t)(kListLen - kChunk)) {
      flush(cnt);
      __syncwarp();
      oa = lbase;
    }
    const uint2 qq = *reinterpret_cast<const uint2 *>(tb + u0 + 4 * q);
    const uint32_t quads[4] = {qq.x & 0xffffu, qq.x >> 16, qq.y & 0xffffu, qq.y >> 16};
    // steps of this chunk that hold a real quad for some lane (warp-uniform)
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
      // the stores are in bounds whether or not they are kept: the check above
      // leaves room for every candidate of this chunk
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
  float fx, fy, fz;
  Acc e0 = 0, e1 = 0, e2 = 0;
  uint32_t e3 = 0;
  if constexpr (kPacked) {
    fx = acc2.fx.x + acc2.fx.y;
    fy = acc2.fy.x + acc2.fy.y;
    fz = acc2.fz.x + acc2.fz.y;
#pragma unroll
    for (int o = 8; o < 32; o <<= 1) {
      fx += __shfl_xor_sync(0xffffffffu, fx, o);
      fy += __shfl_xor_sync(0xffffffffu, fy, o);
      fz += __shfl_xor_sync(0xffffffffu, fz, o);
    }
    if (ENERGY) {
      e0 = acc2.pe.x + acc2.pe.y;
      e1 = acc2.pes.x + acc2.pes.y;
      e2 = acc2.vir.x + acc2.vir.y;
      e3 = acc2.n;
    }
  } else {
    // combine the 4 partial sums of each home atom (lanes il, il+8, il+16, il+24)
#pragma unroll
    for (int o = 8; o < 32; o <<= 1) {
      acc.fx += __shfl_xor_sync(0xffffffffu, acc.fx, o);
      acc.fy += __shfl_xor_sync(0xffffffffu, acc.fy, o);
      acc.fz += __shfl_xor_sync(0xffffffffu, acc.fz, o);
    }
    fx = (float)acc.fx;
    fy = (float)acc.fy;
    fz = (float)acc.fz;
    if (ENERGY) {
      e0 = acc.pe;
      e1 = acc.pes;
      e2 = acc.vir;
      e3 = acc.n;
    }
  }
  if (valid && q == 0) b.F[pi] = make_float4(fx, fy, fz, 0.0f);
  if (ENERGY) {
    ce[0] = warp_sum((double)e0);
    ce[1] = warp_sum((double)e1);
    ce[2] = warp_sum((double)e2);
    ce[3] = (double)warp_sum(e3);
  }
}

// One cluster, one atom type, FP32 sums, LJ or capped law.  Phase 1 tests
// the quads as consume_cluster does but appends a quad, not a candidate: one
// 4-byte entry per quad with at least one admitted candidate, in a per-lane
// list laid out lane-minor (entry k of lane l at 128 k + 4 l, one bank per
// lane).  Phase 2 evaluates the 4 candidates of every listed quad in packed
// FP32x2 and keeps the ones inside the exact cutoff; a far atom of the quad
// (a run's padding) has r^2 = +inf and is dropped by the same test.
template <bool ENERGY, int MODE>
__device__ __forceinline__ void consume_cluster_quads(const ForceBufs &b, const ItemDesc<1> &d,
                                                      const Planes &pl, uint32_t cl,
                                                      uint16_t *mylist, uint16_t *tb,
                                                      double (&ce)[4]) {
  constexpr uint32_t kEntries = kListLen / 2;  // 4-byte entries per lane
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
  const uint32_t pi = valid && q == 0 ? __ldg(b.pid + d.home_g0 + h) : 0u;
  const uint32_t Q = d.Q[cl], M = d.M[cl];
  const uint32_t magic = 0xffffffffu / M + 1u;
  for (uint32_t idx = lane; idx < 9u * M; idx += 32) {
    const uint32_t c = __umulhi(idx, magic), i = idx - c * M;
    if (i < d.len[cl][c]) tb[table_pos(d.pre[cl][c] + i)] = (uint16_t)(d.q0[cl][c] + i);
  }
  for (uint32_t u = Q + lane; u < ((Q + 15u) & ~15u); u += 32)
    tb[table_pos(u)] = (uint16_t)d.sentinel;
  __syncwarp();

  const float rc2 = d.lj.rc2[0];
  const float2 nrc = make_float2(-rc2 * (1.0f + 1.0f / 1024.0f), -rc2 * (1.0f + 1.0f / 1024.0f));
  const float2 m1 = make_float2(-1.0f, -1.0f), two = make_float2(2.0f, 2.0f);
  const float2 half = make_float2(0.5f, 0.5f);
  const float2 s2 = make_float2(d.lj.s2[0], d.lj.s2[0]);
  const float2 e24 = make_float2(d.lj.e24[0], d.lj.e24[0]);
  const float2 e4 = make_float2(d.lj.e4[0], d.lj.e4[0]);
  const float ush = d.lj.ush[0];
  const float2 xi2 = make_float2(xi, xi), yi2 = make_float2(yi, yi), zi2 = make_float2(zi, zi);
  const uint32_t xa = smem_u32(X), ya = smem_u32(Y), za = smem_u32(Z);
  const uint32_t lbase = smem_u32(mylist) + 4u * (uint32_t)lane;
  PairAcc2<ENERGY> a;
  // two candidates of a listed quad: force (and energy) inside the exact cutoff
  auto pair2 = [&](float2 dx, float2 dy, float2 dz) {
    const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
    const bool ina = r2.x < rc2 && r2.x > 0.0f, inb = r2.y < rc2 && r2.y > 0.0f;
    float2 r2c = r2;
    if (MODE == kModeCapped) {
      const float2 fl = __fmul2_rn(make_float2(0.25f, 0.25f), s2);
      r2c = make_float2(fmaxf(r2.x, fl.x), fmaxf(r2.y, fl.y));
    }
    const float2 inv = make_float2(rcp_approx(r2c.x), rcp_approx(r2c.y));
    const float2 sr2 = __fmul2_rn(s2, inv);
    const float2 sr6 = __fmul2_rn(__fmul2_rn(sr2, sr2), sr2);
    const float2 t = __ffma2_rn(two, sr6, m1);
    float2 f = __fmul2_rn(__fmul2_rn(__fmul2_rn(e24, sr6), t), inv);
    f.x = ina ? f.x : 0.0f;
    f.y = inb ? f.y : 0.0f;
    a.fx = __ffma2_rn(f, dx, a.fx);
    a.fy = __ffma2_rn(f, dy, a.fy);
    a.fz = __ffma2_rn(f, dz, a.fz);
    if (ENERGY) {
      float2 u = __fmul2_rn(__fmul2_rn(e4, sr6), __fadd2_rn(sr6, m1));
      u.x = ina ? u.x : 0.0f;
      u.y = inb ? u.y : 0.0f;
      float2 us = __fadd2_rn(u, make_float2(-ush, -ush));
      us.x = ina ? us.x : 0.0f;
      us.y = inb ? us.y : 0.0f;
      a.pe = __ffma2_rn(half, u, a.pe);
      a.pes = __ffma2_rn(half, us, a.pes);
      // f is zero outside the cutoff, where r^2 may be +inf
      float2 w = __fmul2_rn(__fmul2_rn(half, f), r2c);
      w.x = ina ? w.x : 0.0f;
      w.y = inb ? w.y : 0.0f;
      a.vir = __fadd2_rn(a.vir, w);
      a.n += (uint32_t)ina + (uint32_t)inb;
    }
  };
  auto flush = [&](uint32_t cnt) {
    const uint32_t steps = __reduce_max_sync(0xffffffffu, cnt);
    for (uint32_t k = 0; k < steps; ++k) {
      const uint32_t quad = k < cnt ? lds_u32(lbase + 128u * k) : d.sentinel;
      const float4 x4 = lds_f4(xa + quad * 16u), y4 = lds_f4(ya + quad * 16u),
                   z4 = lds_f4(za + quad * 16u);
      pair2(__ffma2_rn(make_float2(x4.x, x4.y), m1, xi2),
            __ffma2_rn(make_float2(y4.x, y4.y), m1, yi2),
            __ffma2_rn(make_float2(z4.x, z4.y), m1, zi2));
      pair2(__ffma2_rn(make_float2(x4.z, x4.w), m1, xi2),
            __ffma2_rn(make_float2(y4.z, y4.w), m1, yi2),
            __ffma2_rn(make_float2(z4.z, z4.w), m1, zi2));
    }
  };
  uint32_t oa = lbase;  // shared-memory address of this lane's next entry
  for (uint32_t u0 = 0; u0 < Q; u0 += kChunk) {
    const uint32_t cnt = (oa - lbase) >> 7;
    if (__reduce_max_sync(0xffffffffu, cnt) > kEntries - kChunk / 4) {
      flush(cnt);
      __syncwarp();
      oa = lbase;
    }
    const uint2 qq = *reinterpret_cast<const uint2 *>(tb + u0 + 4 * q);
    const uint32_t quads[4] = {qq.x & 0xffffu, qq.x >> 16, qq.y & 0xffffu, qq.y >> 16};
    const uint32_t nsteps = min((Q - u0 + 3u) >> 2, (uint32_t)(kChunk / 4));
    // one quad: 4 candidate tests; the quad is stored, and kept when any
    // candidate is admitted (sign bit of r^2 - rc^2 (1 + 2^-10))
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
      const uint32_t any = (__float_as_uint(da.x) | __float_as_uint(da.y) |
                            __float_as_uint(db.x) | __float_as_uint(db.y)) >> 31;
      sts_u32(oa, quad);
      oa += any << 7;
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
  flush((oa - lbase) >> 7);
  __syncwarp();
  float fx = a.fx.x + a.fx.y, fy = a.fy.x + a.fy.y, fz = a.fz.x + a.fz.y;
#pragma unroll
  for (int o = 8; o < 32; o <<= 1) {
    fx += __shfl_xor_sync(0xffffffffu, fx, o);
    fy += __shfl_xor_sync(0xffffffffu, fy, o);
    fz += __shfl_xor_sync(0xffffffffu, fz, o);
  }
  if (valid && q == 0) b.F[pi] = make_float4(fx, fy, fz, 0.0f);
  if (ENERGY) {
    ce[0] = warp_sum((double)(a.pe.x + a.pe.y));
    ce[1] = warp_sum((double)(a.pes.x + a.pes.y));
    ce[2] = warp_sum((double)(a.vir.x + a.vir.y));
    ce[3] = (double)warp_sum(a.n);
  }
}

// Global-memory path of an item whose stage does not fit: task t covers the
// groups of 32 consecutive home atoms t, t + ntask, ...; lanes are atoms.
template <int NT, bool ENERGY, typename Acc, int MODE>
__device__ void consume_task_global(const ForceBufs &b, const ItemDesc<NT> &d, uint32_t t,
                                    double (&ce)[4]) {
  const int lane = threadIdx.x & 31;
  const int nseg = d.nseg, z0 = d.z0, nz = d.nz;
  const uint32_t hbeg = d.off[4][1];
  const uint32_t H = d.H;
  double s[4] = {0.0, 0.0, 0.0, 0.0};
  for (uint32_t gi = t; gi * 32 < H; gi += d.ntask) {
    const uint32_t h = gi * 32 + lane;
    const bool valid = h < H;
    const uint32_t hh = valid ? h : H - 1;
    // home cell (staged index k in [1, nseg]) of this lane, and the warp's span
    int lo = 1, hi = nseg;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (d.off[4][mid] - hbeg <= hh) lo = mid; else hi = mid - 1;
    }
    const int kmin = __reduce_min_sync(0xffffffffu, lo);
    const int kmax = __reduce_max_sync(0xffffffffu, lo);
    const uint32_t gh = d.home_g0 + hh;
    const float4 p = b.rs[gh];
    const float xi = p.x - d.sx[4], yi = p.y - d.sy[4], zi = p.z - d.sz_mid;
    const int ti = NT == 1 ? 0 : __float_as_int(p.w);
    PairAcc<NT, ENERGY, Acc, MODE> acc;
    for (int c = 0; c < 9; ++c) {
      if (!d.periodic && d.kbase[c] == kNoCell) continue;  // no column past an open face
      for (int k = kmin - 1; k <= kmax + 1; ++k) {
        const int zr = z0 - 1 + k, zc = (zr + nz) % nz;
        if (!d.periodic && (zr < 0 || zr >= nz)) continue;
        const uint32_t key = d.kbase[c] + (uint32_t)zc;
        const float sz = k == 0 ? d.sz_lo : (k == nseg + 1 ? d.sz_hi : d.sz_mid);
        if (c == 4)
          global_range<NT, ENERGY, true, Acc, MODE>(b.rs, b.start[key], b.start[key + 1], xi, yi,
                                                    zi, ti, d.sx[c], d.sy[c], sz, gh, d.lj, acc);
        else
          global_range<NT, ENERGY, false, Acc, MODE>(b.rs, b.start[key], b.start[key + 1], xi,
                                                     yi, zi, ti, d.sx[c], d.sy[c], sz, 0, d.lj,
                                                     acc);
      }
    }
    if (valid) b.F[b.pid[gh]] = make_float4((float)acc.fx, (float)acc.fy, (float)acc.fz, 0.0f);
    if (ENERGY) {
      s[0] += warp_sum(valid ? (double)acc.pe : 0.0);
      s[1] += warp_sum(valid ? (double)acc.pes : 0.0);
      s[2] += warp_sum(valid ? (double)acc.vir : 0.0);
      s[3] += (double)warp_sum(valid ? acc.n : 0u);
    }
  }
  for (int k = 0; k < 4; ++k) ce[k] = s[k];
}

// ---- the kernel ---------------------------------------------------------------

template <int NT, bool ENERGY, typename Acc, int kProd, int kCons, int MODE>
__global__ void __launch_bounds__((kProd + kCons) * 32, (kProd + kCons) >= 16 ? 1 : 2)
    k_force(ForceBufs b) {
  pdl_enter();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ ItemDesc<NT> desc[2];
  __shared__ Scratch sc;
  __shared__ uint64_t full[2], empty[2];
  __shared__ double cle[2][kWinCap][4];
  __shared__ int abort_flag, wait_ok;
  __shared__ uint32_t next_item;

  const uint32_t slots = padded_slots((uint32_t)b.cap);
  const uint32_t pbytes = plane_bytes(slots, NT), wbytes = warp_bytes(slots);
  // stage buffer k (computed, not indexed, so it stays in registers)
  auto planes = [&](int k) {
    float *base = reinterpret_cast<float *>(smem_raw + (size_t)k * pbytes);
    Planes p;
    p.X = base;
    p.Y = base + slots;
    p.Z = base + 2 * slots;
    p.T = NT > 1 ? reinterpret_cast<uint32_t *>(base + 3 * slots) : nullptr;
    return p;
  };
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t polls = b.wait_polls ? b.wait_polls : kWaitPolls;
  if (threadIdx.x == 0) {
    for (int k = 0; k < 2; ++k) {
      mbar_init(&full[k], 1);
      mbar_init(&empty[k], kCons);
    }
    abort_flag = 0;
    mbar_fence_init();
  }
  __syncthreads();
  const volatile int *abort_v = &abort_flag;

  if (warp < kProd) {
    // producers: wait for a free buffer (thread 0 polls; the group learns the
    // outcome through its barrier), then stage the next item into it
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
    // Items are claimed from a global counter (queue[0]), so that a CTA that
    // runs faster than the other CTA on its SM takes more of them (the result
    // of an item does not depend on which CTA computes it).  A CTA that will
    // claim no more counts itself in queue[1]; the last one resets both for
    // the next launch.
    auto done_claiming = [&]() {
      if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(b.queue + 1, 1u) == gridDim.x - 1) {
          atomicExch(b.queue, 0u);
          atomicExch(b.queue + 1, 0u);
        }
      }
    };
    uint32_t running = 0;
    uint32_t n = 0;
    for (;; ++n) {
      if (threadIdx.x == 0) next_item = atomicAdd(b.queue, 1u);
      const int bf = n & 1;
      if (n >= 2) {
        // the consumers are done with item n - 2 in this buffer
        if (!wait_empty(bf, ((n >> 1) - 1) & 1u)) {
          done_claiming();
          return;
        }
        if (ENERGY && threadIdx.x == 0) write_partials(b, desc[bf], cle[bf]);
      }
      producer_sync<kProd>();
      const uint32_t item = next_item;
      producer_sync<kProd>();
      if (item >= b.nitems) {
        // no item left: an end marker in this buffer stops the consumers
        done_claiming();
        if (threadIdx.x == 0) {
          desc[bf].item = kNone;
          mbar_arrive(&full[bf]);
        }
        break;
      }
      const bool ok = produce_item<NT, MODE, kProd, kCons>(
          b, item, desc[bf], sc, planes(bf), running);
      if (!ok) {
        done_claiming();
        if (threadIdx.x == 0) abort_flag = 1;
        return;
      }
      // test hook (failure-detection test entry only): withhold the first
      // hand-off so that the consumers' bounded wait runs out
      const bool withhold = (b.test_flags & 1u) && n == 0;
      if (threadIdx.x == 0 && !withhold) mbar_arrive(&full[bf]);
    }
    // the last item: wait for the consumers, then its energy partials
    if (n >= 1) {
      const uint32_t m = n - 1;
      const int bf = m & 1;
      if (!wait_empty(bf, (m >> 1) & 1u)) return;
      if (ENERGY && threadIdx.x == 0) write_partials(b, desc[bf], cle[bf]);
    }
    return;
  }

  // consumers
  const int cw = warp - kProd;
  uint16_t *mylist =
      reinterpret_cast<uint16_t *>(smem_raw + 2 * (size_t)pbytes + (size_t)cw * wbytes);
  uint16_t *tb = mylist + 32 * kListLen;
  for (uint32_t n = 0;; ++n) {
    const int bf = n & 1;
    bool ok = lane != 0 || mbar_wait_or_abort(&full[bf], (n >> 1) & 1u, abort_v, polls);
    ok = __shfl_sync(0xffffffffu, ok, 0);
    if (!ok) {
      if (lane == 0 && !*abort_v) atomicOr(&b.status[0], kStatusWaitTimeout);
      return;
    }
    const ItemDesc<NT> &d = desc[bf];
    if (d.item == kNone) break;  // end marker
    const Planes pbuf = planes(bf);
    if (!d.skip) {
      if (!d.overflow) {
        // clusters go round-robin over the CTA's whole item sequence
        const uint32_t first = ((uint32_t)cw + (uint32_t)kCons - d.base) % (uint32_t)kCons;
        for (uint32_t cl = first; cl < d.nclus; cl += kCons) {
          double ce[4];
          if constexpr (NT == 1 && std::is_same<Acc, float>::value && MODE != kModeSoftCore)
            consume_cluster_quads<ENERGY, MODE>(b, d, pbuf, cl, mylist, tb, ce);
          else
            consume_cluster<NT, ENERGY, Acc, MODE>(b, d, pbuf, cl, mylist, tb, ce);
          if (ENERGY && lane == 0)
            for (int k = 0; k < 4; ++k) cle[bf][cl][k] = ce[k];
        }
      } else {
        for (uint32_t t = (uint32_t)cw; t < d.ntask; t += kCons) {
          double ce[4];
          consume_task_global<NT, ENERGY, Acc, MODE>(b, d, t, ce);
          if (ENERGY && lane == 0)
            for (int k = 0; k < 4; ++k) cle[bf][t][k] = ce[k];
        }
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[bf]);
  }
}

// CTAs per SM of a launch shape, from the occupancy calculator.
template <typename K>
int resident_ctas(K kern, int threads, size_t smem) {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, threads, smem) != cudaSuccess) n = 1;
  return n > 0 ? n : 1;
}

int sm_count() {
  static int n = 0;
  if (n == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 1;
  }
  return n;
}

template <int NT, bool E, typename Acc, int P, int C, int MODE = kModeLJ>
cudaError_t launch_w(const ForceBufs &b, cudaStream_t s) {
  const size_t smem = smem_bytes((uint32_t)b.cap, C, NT);
  auto kern = k_force<NT, E, Acc, P, C, MODE>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  // persistent grid: every resident CTA slot, at most one CTA per item
  const long slots = (long)resident_ctas(kern, (P + C) * 32, smem) * sm_count();
  const unsigned grid = (unsigned)std::min<long>(slots, (long)b.nitems);
  return launch_pdl(kern, dim3(grid), dim3((P + C) * 32), smem, s, b);
}

// Launch shapes (producer warps, consumer warps): the default, and a small one.
constexpr int kProdDefault = 4, kConsDefault = 8;
constexpr int kProdSmall = 2, kConsSmall = 4;

template <int NT, bool E, typename Acc>
cudaError_t launch_t(const ForceBufs &b, int threads, cudaStream_t s) {
  return threads == 128 ? launch_w<NT, E, Acc, kProdSmall, kConsSmall>(b, s)
                        : launch_w<NT, E, Acc, kProdDefault, kConsDefault>(b, s);
}

template <int NT>
cudaError_t launch_nt(const ForceBufs &b, bool energy, bool acc64, int threads, cudaStream_t s) {
  if (energy) {
    return acc64 ? launch_t<NT, true, double>(b, threads, s)
                 : launch_t<NT, true, float>(b, threads, s);
  }
  return acc64 ? launch_t<NT, false, double>(b, threads, s)
               : launch_t<NT, false, float>(b, threads, s);
}

template <int MODE>
cudaError_t launch_mode(const ForceBufs &b, int nt_max, cudaStream_t s) {
  if (b.nitems == 0) return cudaSuccess;
  switch (nt_max) {
    case 1: return launch_w<1, false, float, kProdDefault, kConsDefault, MODE>(b, s);
    case 2: return launch_w<2, false, float, kProdDefault, kConsDefault, MODE>(b, s);
    case 3: case 4: return launch_w<4, false, float, kProdDefault, kConsDefault, MODE>(b, s);
    default: return launch_w<8, false, float, kProdDefault, kConsDefault, MODE>(b, s);
  }
}

}  // namespace

int force_max_segment() { return kMaxSeg; }

int force_max_capacity(int warps, int nt) {
  // largest staged-atom capacity whose shared memory fits one CTA
  const int consumers = warps >= 8 ? kConsDefault : kConsSmall;
  (void)kProdSmall;
  uint32_t cap = 64;
  while (smem_bytes(cap + 64, consumers, nt) <= 180u * 1024u) cap += 64;
  return (int)cap;
}

// Static shared memory of a force CTA for up to `nt` types: the two item
// descriptors, the producer scratch, the per-cluster energy sums, and 1 KB
// for barriers and flags.
template <int NT>
constexpr uint32_t static_smem() {
  return 2u * (uint32_t)sizeof(ItemDesc<NT>) + (uint32_t)sizeof(Scratch) +
         2u * kWinCap * 4u * 8u + 1024u;
}

int force_smem_per_cta(int cap, int nt) {
  const uint32_t st = nt <= 1 ? static_smem<1>() : nt <= 2 ? static_smem<2>()
                      : nt <= 4 ? static_smem<4>() : static_smem<8>();
  return (int)(smem_bytes((uint32_t)cap, kConsDefault, nt) + st);
}

int force_smem_limit() {
  // two CTAs per SM share its 228 KB, less 1 KB per CTA reserved by the driver
  return 112 * 1024;
}

int force_threads() { return 256; }

cudaError_t launch_force_capped(const ForceBufs &b, int nt_max, cudaStream_t s) {
  return launch_mode<kModeCapped>(b, nt_max, s);
}

cudaError_t launch_force_softcore(const ForceBufs &b, int nt_max, cudaStream_t s) {
  return launch_mode<kModeSoftCore>(b, nt_max, s);
}

cudaError_t launch_force(const ForceBufs &b, int nt_max, bool energy, bool acc64,
                         int block_threads, cudaStream_t s) {
  if (b.nitems == 0) return cudaSuccess;
  switch (nt_max) {
    case 1: return launch_nt<1>(b, energy, acc64, block_threads, s);
    case 2: return launch_nt<2>(b, energy, acc64, block_threads, s);
    case 3: case 4: return launch_nt<4>(b, energy, acc64, block_threads, s);
    default: return launch_nt<8>(b, energy, acc64, block_threads, s);
  }
}

}  // namespace pb
