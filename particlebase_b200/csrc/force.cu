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
// Work decomposition.  One CTA per work item = (system, x-y column of cells,
// run of z cells [z0, z1)).  The CTA stages the 3 x 3 neighbour columns over
// z cells [z0 - 1, z1] (periodic halo cells included) into shared memory with
// 1-D bulk copies (cp.async.bulk, mbarrier completion, no multicast).
//
// Coordinate frame.  Positions are absolute FP32 coordinates.  Each CTA moves
// all staged atoms into one frame by subtracting 0 or L per axis: a neighbour
// image below the box (atoms near the top face) and, in CTAs on the top face,
// every non-wrapped atom, get x - L.  The subtraction only ever applies to
// coordinates >= L/2, where it is exact (Sterbenz), so displacements x_i - x_j
// in the frame are the minimum-image displacements with no rounding beyond
// the subtraction itself, even in a 190-sigma box.  Work items are laid out
// so that a top-face item's cells all lie above the box middle.
//
// Stage layout.  The bulk copies land the 9 staged columns as float4 (x, y,
// z, type bits) in a landing zone, each column starting at a multiple of 4
// slots.  One pass applies the frame shift and writes structure-of-arrays
// planes X, Y, Z (and a type plane) in the same padded slot order; the pad
// slots of each column hold a far sentinel, so every column is a whole number
// of 4-atom quads.  The landing zone is then reused for the pair lists.
//
// Compute (shared-memory path).  Cells are sorted by z and atoms within a
// cell by z, so every staged column is one z-sorted array.  A warp takes a
// cluster of 8 consecutive home atoms (lane & 7) and splits the candidates 4
// ways (lane >> 3).  Lanes binary-search the z window [z_min - rc, z_max + rc]
// of the cluster in each of the 9 columns, round it out to whole quads and
// write the quads of all 9 windows into one per-warp table, so the candidate
// loop runs over one flat sequence with no per-column tails.  Then
//   phase 1  tests 4 candidates per step (one quad, packed FP32x2 arithmetic)
//            against rc^2 (1 + 2^-10) and appends the hits to a per-lane index
//            list in shared memory (no divergent force code);
//   phase 2  recomputes each listed pair exactly, applies the exact cutoff
//            r^2 < rc^2 of the pair's types (which also drops the self pair,
//            r^2 = 0), and evaluates the force, two list entries per step in
//            packed FP32x2 arithmetic.
// The 4 partial sums of an atom are combined with two warp shuffles.
// A CTA whose stage would exceed its shared-memory capacity computes from
// global memory instead (slower, same result) and raises a status bit.
#include <type_traits>

#include "md.cuh"
#include "tma.cuh"

namespace pb {
namespace {

constexpr int kMaxSeg = 40;     // longest z run of one work item (cells)
constexpr int kDefaultWarps = 8;
constexpr int kListLen = 48;    // per-lane pair list entries
constexpr int kChunk = 16;      // candidates a lane tests between list checks
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

struct Stage {
  // index within column c of the first staged atom of z cell k (k = 0 is image
  // cell z0 - 1, k = nseg + 1 is image cell z1); entry nseg + 2 is the column's count
  uint32_t off[9][kMaxSeg + 3];
  uint32_t ps[10];     // first padded slot of each column (multiples of 4); ps[9] = total
  uint32_t kbase[9];   // packed key of z cell 0 of each column
  float sx[9], sy[9];  // frame shift of each column (0 or L)
  float sz_lo, sz_mid, sz_hi;  // frame shift of staged cell 0, 1..nseg, nseg + 1
  uint64_t bar;
  uint32_t total;
  uint32_t home_g0;    // global sorted index of the first home atom
  int overflow;
};

// Padded slots for `cap` staged atoms: each of the 9 columns rounds up to a
// multiple of 4 (at most 3 pad slots per column), plus one quad of far atoms
// that pads the last chunk of every quad table.
__host__ __device__ __forceinline__ uint32_t padded_slots(uint32_t cap) {
  return ((cap + 27u + 3u) & ~3u) + 4u;
}

// z windows of a batch of clusters: first quad, quads and flat offset of the
// window of each (cluster, column), and per cluster the total and the longest.
constexpr int kWinCap = 64;
struct Windows {
  uint16_t q0[kWinCap][9], len[kWinCap][9], pre[kWinCap][9];
  uint16_t Q[kWinCap], M[kWinCap];
};

// Bytes of one warp's pair lists plus its quad table (at most one entry per
// padded quad of the stage).
__host__ __device__ __forceinline__ uint32_t warp_bytes(uint32_t slots) {
  return ((32u * kListLen * 2u + (slots / 4u + kChunk) * 2u) + 15u) & ~15u;
}

// Position of flat quad u in a warp's quad table: within each chunk of 16,
// the 4 quads lane q tests (u = q, q + 4, q + 8, q + 12) are adjacent, so a
// lane fetches a chunk's quads with one 8-byte load.
__device__ __forceinline__ uint32_t table_pos(uint32_t u) {
  return (u & ~15u) | ((u & 3u) << 2) | ((u >> 2) & 3u);
}

// Dynamic shared memory of one CTA: the landing zone (reused for the lists)
// followed by the X, Y, Z planes and, with more than one type, the type plane.
__host__ __device__ __forceinline__ uint32_t smem_bytes(uint32_t cap, int warps, int nt) {
  const uint32_t slots = padded_slots(cap);
  const uint32_t land = slots * 16u, lists = (uint32_t)warps * warp_bytes(slots);
  const uint32_t zone = land > lists ? land : lists;
  const uint32_t planes = (slots * 12u + (nt > 1 ? slots : 0u) + 15u) & ~15u;
  return zone + planes;
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

// Phase 2, general form: one listed pair per step, any force law and any
// accumulator type.  Entries are padded slots; the exact cutoff drops the
// candidates phase 1 admitted through its margin and the self pair.
template <int NT, bool ENERGY, typename Acc, int MODE>
__device__ __forceinline__ void flush_scalar(const float *X, const float *Y, const float *Z,
                                             const uint8_t *T, const uint16_t *list,
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
                                             const uint8_t *T, const uint16_t *list,
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
  for (uint32_t k = 0; k < cnt; k += 2) {
    const uint32_t j0 = list[k * 32 + lane];
    const uint32_t j1 = list[min(k + 1, cnt - 1) * 32 + lane];
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
    const float2 dx = __ffma2_rn(make_float2(X[j0], X[j1]), m1, xi2);
    const float2 dy = __ffma2_rn(make_float2(Y[j0], Y[j1]), m1, yi2);
    const float2 dz = __ffma2_rn(make_float2(Z[j0], Z[j1]), m1, zi2);
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

template <int NT, bool ENERGY, typename Acc, int kWarps, int MODE>
__global__ void __launch_bounds__(kWarps * 32, 24 / kWarps) k_force(ForceBufs b) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ Stage st;
  __shared__ LJLocal<NT> ljs;
  __shared__ uint32_t cnt_cell[9][kMaxSeg + 3];
  __shared__ uint32_t gstart[9][kMaxSeg + 3];
  __shared__ Windows win;
  __shared__ double red[4 * 32];
  // packed phase 2 for FP32 sums of the LJ and capped laws
  constexpr bool kPacked = std::is_same<Acc, float>::value && MODE != kModeSoftCore;

  const uint32_t slots = padded_slots((uint32_t)b.cap);
  const uint32_t land_bytes = slots * 16u, wbytes = warp_bytes(slots);
  const uint32_t zone = land_bytes > kWarps * wbytes ? land_bytes : kWarps * wbytes;
  float4 *land = reinterpret_cast<float4 *>(smem_raw);
  float *X = reinterpret_cast<float *>(smem_raw + zone);
  float *Y = X + slots;
  float *Z = Y + slots;
  uint8_t *T = reinterpret_cast<uint8_t *>(Z + slots);

  const ForceItem it = b.items[blockIdx.x];
  if (b.steps_left != nullptr && b.steps_left[it.sys] == 0) {
    // a system whose step budget is spent keeps its state; nothing to compute
    if (ENERGY && threadIdx.x < 4) b.partials[(size_t)blockIdx.x * 4 + threadIdx.x] = 0.0;
    return;
  }
  const SysDesc &S = b.sys[it.sys];
  const Grid g = S.g;
  const int nx = g.n[0], ny = g.n[1], nz = g.n[2];
  const int z0 = it.z0, z1 = it.z1, nseg = z1 - z0;
  const int ncell = nseg + 2;  // staged cells per column
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

  if (threadIdx.x < NT * NT) {
    const LJTable &Tb = b.lj[S.lj];
    const int a = threadIdx.x / NT, c = threadIdx.x % NT;
    const int k = a * Tb.nt + c;
    ljs.s2[threadIdx.x] = Tb.s2[k];
    ljs.e24[threadIdx.x] = Tb.e24[k];
    ljs.e4[threadIdx.x] = Tb.e4[k];
    ljs.rc2[threadIdx.x] =
        MODE == kModeSoftCore ? fminf(Tb.rc2[k], b.sc_rc * b.sc_rc) : Tb.rc2[k];
    ljs.ush[threadIdx.x] = Tb.ushift[k];
  }
  if (threadIdx.x == 0) {
    ljs.sc_rc = b.sc_rc;
    ljs.sc_f0 = b.sc_f0;
  }
  if (threadIdx.x < 9) {
    const int cx = it.cx, cy = it.cy;
    const int c = threadIdx.x;
    const int ax = cx + c / 3 - 1, ay = cy + c % 3 - 1;
    const int wx = ax < 0 ? -1 : (ax >= nx ? 1 : 0);
    const int wy = ay < 0 ? -1 : (ay >= ny ? 1 : 0);
    // frame: F = L on the top face; staged = x + w L - F, so the shift is F - w L
    const float Fx = cx == nx - 1 ? g.L[0] : 0.0f, Fy = cy == ny - 1 ? g.L[1] : 0.0f;
    st.sx[c] = Fx - (float)wx * g.L[0];
    st.sy[c] = Fy - (float)wy * g.L[1];
    st.kbase[c] = it.kbase[c];
  }
  if (threadIdx.x == 0) {
    const float Fz = z1 == nz ? g.L[2] : 0.0f;
    st.sz_lo = z0 == 0 ? Fz + g.L[2] : Fz;   // image z0 - 1 wraps below when z0 == 0
    st.sz_mid = Fz;
    st.sz_hi = z1 == nz ? Fz - g.L[2] : Fz;  // image z1 wraps above when z1 == nz
  }
  // counts of the 9 x ncell staged cells, one per thread; cell starts kept
  for (int t = threadIdx.x; t < 9 * ncell; t += blockDim.x) {
    const int c = t / ncell, k = t % ncell;
    const int zc = (z0 - 1 + k + nz) % nz;
    const uint32_t key = it.kbase[c] + (uint32_t)zc;
    const uint32_t s0 = b.start[key];
    gstart[c][k] = s0;
    cnt_cell[c][k] = b.start[key + 1] - s0;
  }
  __syncthreads();
  // exclusive prefix over the cells of each column, one warp per column
  for (int c = warp; c < 9; c += kWarps) {
    uint32_t run = 0;
    for (int base = 0; base < ncell; base += 32) {
      const int k = base + lane;
      const uint32_t v = k < ncell ? cnt_cell[c][k] : 0u;
      uint32_t incl = v;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
      }
      if (k < ncell) st.off[c][k] = run + incl - v;
      run += __shfl_sync(0xffffffffu, incl, 31);
    }
    if (lane == 0) st.off[c][ncell] = run;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t p = 0, run = 0;
    for (int c = 0; c < 9; ++c) {
      const uint32_t n = st.off[c][ncell];
      st.ps[c] = p;
      p += (n + 3u) & ~3u;
      run += n;
    }
    st.ps[9] = p;
    st.total = run;
    // the system's own capacity decides: the same path alone or batched
    // (4 slots stay free for the sentinel quad)
    st.overflow = p + 4u > padded_slots(S.cap);
    st.home_g0 = gstart[4][1];
    if (!st.overflow && run > 0) {
      mbar_init(&st.bar, 9);
      mbar_fence_init();
    }
  }
  __syncthreads();
  const bool overflow = st.overflow;
  if (!overflow && st.total > 0) {
    if (threadIdx.x < 9) {
      // column c: up to three contiguous runs (below halo, main, above halo)
      const int c = threadIdx.x;
      const uint32_t base = st.ps[c];
      mbar_arrive_expect_tx(&st.bar, st.off[c][ncell] * 16u);
      int k = 0;
      while (k < ncell) {
        const int zc = (z0 - 1 + k + nz) % nz;
        int kend = k;
        while (kend + 1 < ncell && ((z0 - 1 + kend + 1 + nz) % nz) == zc + (kend + 1 - k)) ++kend;
        const uint32_t g0 = gstart[c][k];
        const uint32_t g1 = gstart[c][kend] + cnt_cell[c][kend];
        if (g1 > g0) bulk_g2s(&land[base + st.off[c][k]], &b.rs[g0], (g1 - g0) * 16u, &st.bar);
        k = kend + 1;
      }
    }
    // one thread polls the barrier; the others sleep at the CTA barrier and
    // see the copied data through it
    const bool ok = threadIdx.x != 0 || mbar_wait_bounded(&st.bar, 0);
    if (__syncthreads_or(!ok)) {
      // give the copies in flight a second bounded wait before the CTA leaves
      if (threadIdx.x == 0) {
        atomicOr(&b.status[it.sys], kStatusWaitTimeout);
        mbar_wait_bounded(&st.bar, 0);
      }
      return;
    }
    // frame shift and SoA planes; pad slots get the far sentinel
    for (int c = 0; c < 9; ++c) {
      const uint32_t p0 = st.ps[c], p1 = st.ps[c + 1];
      const uint32_t n = st.off[c][ncell];
      const uint32_t lo_end = st.off[c][1];
      const uint32_t hi_beg = st.off[c][nseg + 1];
      const float sx = st.sx[c], sy = st.sy[c];
      for (uint32_t s = p0 + threadIdx.x; s < p1; s += blockDim.x) {
        const uint32_t r = s - p0;
        float x = kFar, y = kFar, z = kFar;
        uint8_t ty = 0;
        if (r < n) {
          const float4 p = land[s];
          const float sz = r < lo_end ? st.sz_lo : (r < hi_beg ? st.sz_mid : st.sz_hi);
          x = p.x - sx;
          y = p.y - sy;
          z = p.z - sz;
          ty = (uint8_t)__float_as_int(p.w);
        }
        X[s] = x;
        Y[s] = y;
        Z[s] = z;
        if (NT > 1) T[s] = ty;
      }
    }
    if (threadIdx.x < 4) {  // the sentinel quad that pads the last chunk of a table
      const uint32_t s = st.ps[9] + threadIdx.x;
      X[s] = kFar;
      Y[s] = kFar;
      Z[s] = kFar;
      if (NT > 1) T[s] = 0;
    }
    __syncthreads();  // the landing zone is free from here on
  } else if (overflow && threadIdx.x == 0) {
    atomicOr(&b.status[it.sys], kStatusSmemOverflow);
  }

  Acc pe = 0, pes = 0, vir = 0;
  uint32_t npairs = 0;

  if (!overflow && st.total > 0) {
    const uint32_t H = st.off[4][nseg + 1] - st.off[4][1];
    const uint32_t hb = st.ps[4] + st.off[4][1];  // slot of home atom 0
    const uint32_t sentinel = st.ps[9] / 4u;       // quad of far atoms
    uint16_t *mylist = reinterpret_cast<uint16_t *>(smem_raw + (size_t)warp * wbytes);
    uint16_t *tb = mylist + 32 * kListLen;
    const int il = lane & 7, q = lane >> 3;
    float rcmax2 = 0.f;
    for (int k = 0; k < NT * NT; ++k) rcmax2 = fmaxf(rcmax2, ljs.rc2[k]);
    const float rcw = sqrtf(rcmax2) * 1.00001f + 1e-5f;
    // phase-1 bound with a margin: a superset of the exact test of phase 2
    const float2 nrc = make_float2(-rcmax2 * (1.0f + 1.0f / 1024.0f),
                                   -rcmax2 * (1.0f + 1.0f / 1024.0f));
    const float2 m1 = make_float2(-1.0f, -1.0f);
    const float4 *X4 = reinterpret_cast<const float4 *>(X);
    const float4 *Y4 = reinterpret_cast<const float4 *>(Y);
    const float4 *Z4 = reinterpret_cast<const float4 *>(Z);
    const uint32_t nclus = (H + 7) / 8;
    for (uint32_t cb = 0; cb < nclus; cb += kWinCap) {
      const uint32_t nb = min((uint32_t)kWinCap, nclus - cb);
      // z windows of every (cluster, column) of this batch, one per thread
      for (uint32_t t = threadIdx.x; t < 9u * nb; t += blockDim.x) {
        const uint32_t k = t / 9u, c = t - 9u * k;
        const uint32_t cl = cb + k;
        const float zmin = Z[hb + cl * 8];
        const float zmax = Z[hb + min(cl * 8 + 7, H - 1)];
        const uint32_t lo = st.ps[c], hi = lo + st.off[c][ncell];
        const uint32_t a = lower_bound_z(Z, lo, hi, zmin - rcw) >> 2;
        const uint32_t e = (upper_bound_z(Z, lo, hi, zmax + rcw) + 3u) >> 2;
        win.q0[k][c] = (uint16_t)a;
        // empty unless ordered (an unsorted column, e.g. NaN positions, can
        // invert the two searches)
        win.len[k][c] = (uint16_t)(e > a ? e - a : 0u);
      }
      __syncthreads();
      for (uint32_t k = threadIdx.x; k < nb; k += blockDim.x) {
        uint32_t s = 0, m = 2;
        for (int c = 0; c < 9; ++c) {
          win.pre[k][c] = (uint16_t)s;
          s += win.len[k][c];
          m = max(m, (uint32_t)win.len[k][c]);
        }
        win.Q[k] = (uint16_t)s;
        win.M[k] = (uint16_t)m;
      }
      __syncthreads();
      for (uint32_t k = warp; k < nb; k += kWarps) {
        const uint32_t cl = cb + k;
        const uint32_t h = cl * 8 + il;
        const bool valid = h < H;
        const uint32_t hs = hb + (valid ? h : H - 1);
        const float xi = valid ? X[hs] : kNoAtom;
        const float yi = valid ? Y[hs] : kNoAtom;
        const float zi = valid ? Z[hs] : kNoAtom;
        const int ti = NT == 1 ? 0 : (int)T[hs];
        // the warp's quad table: lanes cover (column, index) pairs, column =
        // idx / M by a multiply-high (exact while 9 M^2 < 2^32)
        const uint32_t Q = win.Q[k], M = win.M[k];
        const uint32_t magic = 0xffffffffu / M + 1u;
        for (uint32_t idx = lane; idx < 9u * M; idx += 32) {
          const uint32_t c = __umulhi(idx, magic), i = idx - c * M;
          if (i < win.len[k][c]) tb[table_pos(win.pre[k][c] + i)] = (uint16_t)(win.q0[k][c] + i);
        }
        for (uint32_t u = Q + lane; u < ((Q + 15u) & ~15u); u += 32)
          tb[table_pos(u)] = (uint16_t)sentinel;
        __syncwarp();

        PairAcc<NT, ENERGY, Acc, MODE> acc;
        PairAcc2<ENERGY> acc2;
        auto flush = [&](uint32_t cnt) {
          if constexpr (kPacked) {
            flush_packed<NT, ENERGY, MODE>(X, Y, Z, T, mylist, cnt, lane, xi, yi, zi, ti, ljs,
                                           acc2);
          } else {
            flush_scalar<NT, ENERGY, Acc, MODE>(X, Y, Z, T, mylist, cnt, lane, xi, yi, zi, ti,
                                                ljs, acc);
          }
        };
        const float2 xi2 = make_float2(xi, xi), yi2 = make_float2(yi, yi), zi2 = make_float2(zi, zi);
        uint16_t *out = mylist + lane;
        // lane q tests quads u = q, q + 4, ... of the flat sequence, 4 per
        // chunk; the table pads the last chunk with the sentinel quad
        for (uint32_t u0 = 0; u0 < Q; u0 += kChunk) {
          const uint32_t cnt = (uint32_t)(out - (mylist + lane)) >> 5;
          if (__reduce_max_sync(0xffffffffu, cnt) > (uint32_t)(kListLen - kChunk)) {
            flush(cnt);
            __syncwarp();
            out = mylist + lane;
          }
          const uint2 qq = *reinterpret_cast<const uint2 *>(tb + u0 + 4 * q);
          const uint32_t quads[4] = {qq.x & 0xffffu, qq.x >> 16, qq.y & 0xffffu, qq.y >> 16};
#pragma unroll
          for (int kk = 0; kk < kChunk / 4; ++kk) {
            const uint32_t quad = quads[kk];
            const float4 x4 = X4[quad], y4 = Y4[quad], z4 = Z4[quad];
            const float2 dxa = __ffma2_rn(make_float2(x4.x, x4.y), m1, xi2);
            const float2 dxb = __ffma2_rn(make_float2(x4.z, x4.w), m1, xi2);
            const float2 dya = __ffma2_rn(make_float2(y4.x, y4.y), m1, yi2);
            const float2 dyb = __ffma2_rn(make_float2(y4.z, y4.w), m1, yi2);
            const float2 dza = __ffma2_rn(make_float2(z4.x, z4.y), m1, zi2);
            const float2 dzb = __ffma2_rn(make_float2(z4.z, z4.w), m1, zi2);
            const float2 da =
                __ffma2_rn(dza, dza, __ffma2_rn(dya, dya, __ffma2_rn(dxa, dxa, nrc)));
            const float2 db =
                __ffma2_rn(dzb, dzb, __ffma2_rn(dyb, dyb, __ffma2_rn(dxb, dxb, nrc)));
            // the stores are in bounds whether or not they are kept: the check
            // above leaves room for every candidate of this chunk
            const uint32_t s = quad * 4u;
            out[0] = (uint16_t)s;
            out += da.x < 0.0f ? 32 : 0;
            out[0] = (uint16_t)(s + 1u);
            out += da.y < 0.0f ? 32 : 0;
            out[0] = (uint16_t)(s + 2u);
            out += db.x < 0.0f ? 32 : 0;
            out[0] = (uint16_t)(s + 3u);
            out += db.y < 0.0f ? 32 : 0;
          }
        }
        flush((uint32_t)(out - (mylist + lane)) >> 5);
        __syncwarp();
        float fx, fy, fz;
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
            pe += (Acc)(acc2.pe.x + acc2.pe.y);
            pes += (Acc)(acc2.pes.x + acc2.pes.y);
            vir += (Acc)(acc2.vir.x + acc2.vir.y);
            npairs += acc2.n;
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
            pe += acc.pe;
            pes += acc.pes;
            vir += acc.vir;
            npairs += acc.n;
          }
        }
        if (valid && q == 0) {
          const uint32_t gh = st.home_g0 + h;
          b.F[b.pid[gh]] = make_float4(fx, fy, fz, 0.0f);
        }
      }
      __syncthreads();  // the next batch reuses the window arrays
    }
  } else if (overflow) {
    // Global-memory path: 32 consecutive home atoms per warp, one per lane.
    const uint32_t hbeg = st.off[4][1];
    const uint32_t H = st.off[4][nseg + 1] - hbeg;
    for (uint32_t t = warp; t * 32 < H; t += kWarps) {
      const uint32_t h = t * 32 + lane;
      const bool valid = h < H;
      const uint32_t hh = valid ? h : H - 1;
      // home cell (staged index k in [1, nseg]) of this lane, and the warp's span
      int lo = 1, hi = nseg;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (st.off[4][mid] - hbeg <= hh) lo = mid; else hi = mid - 1;
      }
      const int kmin = __reduce_min_sync(0xffffffffu, lo);
      const int kmax = __reduce_max_sync(0xffffffffu, lo);
      const uint32_t gh = st.home_g0 + hh;
      const float4 p = b.rs[gh];
      const float xi = p.x - st.sx[4], yi = p.y - st.sy[4], zi = p.z - st.sz_mid;
      const int ti = NT == 1 ? 0 : __float_as_int(p.w);
      PairAcc<NT, ENERGY, Acc, MODE> acc;
      for (int c = 0; c < 9; ++c) {
        for (int k = kmin - 1; k <= kmax + 1; ++k) {
          const int zc = (z0 - 1 + k + nz) % nz;
          const uint32_t key = st.kbase[c] + (uint32_t)zc;
          const float sz = k == 0 ? st.sz_lo : (k == nseg + 1 ? st.sz_hi : st.sz_mid);
          if (c == 4)
            global_range<NT, ENERGY, true, Acc, MODE>(b.rs, b.start[key], b.start[key + 1], xi, yi,
                                                      zi, ti, st.sx[c], st.sy[c], sz, gh, ljs, acc);
          else
            global_range<NT, ENERGY, false, Acc, MODE>(b.rs, b.start[key], b.start[key + 1], xi,
                                                       yi, zi, ti, st.sx[c], st.sy[c], sz, 0, ljs,
                                                       acc);
        }
      }
      if (valid) {
        b.F[b.pid[gh]] = make_float4((float)acc.fx, (float)acc.fy, (float)acc.fz, 0.0f);
        if (ENERGY) {
          pe += acc.pe;
          pes += acc.pes;
          vir += acc.vir;
          npairs += acc.n;
        }
      }
    }
  }
  if (ENERGY) {
    double v[4] = {(double)pe, (double)pes, (double)vir, (double)npairs};
    block_sum<4>(v, red);
    if (threadIdx.x == 0) {
      b.partials[(size_t)blockIdx.x * 4 + 0] = v[0];
      b.partials[(size_t)blockIdx.x * 4 + 1] = v[1];
      b.partials[(size_t)blockIdx.x * 4 + 2] = v[2];
      b.partials[(size_t)blockIdx.x * 4 + 3] = v[3];
    }
  }
}

template <int NT, bool E, typename Acc, int W, int MODE = kModeLJ>
cudaError_t launch_w(const ForceBufs &b, cudaStream_t s) {
  const size_t smem = smem_bytes((uint32_t)b.cap, W, NT);
  auto kern = k_force<NT, E, Acc, W, MODE>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  kern<<<b.nitems, W * 32, smem, s>>>(b);
  return cudaGetLastError();
}

template <int NT, bool E, typename Acc>
cudaError_t launch_t(const ForceBufs &b, int warps, cudaStream_t s) {
  return warps == 4 ? launch_w<NT, E, Acc, 4>(b, s) : launch_w<NT, E, Acc, 8>(b, s);
}

template <int NT>
cudaError_t launch_nt(const ForceBufs &b, bool energy, bool acc64, int warps, cudaStream_t s) {
  if (energy) {
    return acc64 ? launch_t<NT, true, double>(b, warps, s) : launch_t<NT, true, float>(b, warps, s);
  }
  return acc64 ? launch_t<NT, false, double>(b, warps, s) : launch_t<NT, false, float>(b, warps, s);
}

template <int MODE>
cudaError_t launch_mode(const ForceBufs &b, int nt_max, cudaStream_t s) {
  if (b.nitems == 0) return cudaSuccess;
  switch (nt_max) {
    case 1: return launch_w<1, false, float, kDefaultWarps, MODE>(b, s);
    case 2: return launch_w<2, false, float, kDefaultWarps, MODE>(b, s);
    case 3: case 4: return launch_w<4, false, float, kDefaultWarps, MODE>(b, s);
    default: return launch_w<8, false, float, kDefaultWarps, MODE>(b, s);
  }
}

}  // namespace

int force_max_segment() { return kMaxSeg; }

int force_max_capacity(int warps, int nt) {
  // largest staged-atom capacity whose shared memory fits beside the static part
  uint32_t cap = 64;
  while (smem_bytes(cap + 64, warps, nt) <= 200u * 1024u) cap += 64;
  return (int)cap;
}
int force_threads() { return kDefaultWarps * 32; }

cudaError_t launch_force_capped(const ForceBufs &b, int nt_max, cudaStream_t s) {
  return launch_mode<kModeCapped>(b, nt_max, s);
}

cudaError_t launch_force_softcore(const ForceBufs &b, int nt_max, cudaStream_t s) {
  return launch_mode<kModeSoftCore>(b, nt_max, s);
}

cudaError_t launch_force(const ForceBufs &b, int nt_max, bool energy, bool acc64,
                         int block_threads, cudaStream_t s) {
  if (b.nitems == 0) return cudaSuccess;
  const int warps = block_threads == 128 ? 4 : 8;
  switch (nt_max) {
    case 1: return launch_nt<1>(b, energy, acc64, warps, s);
    case 2: return launch_nt<2>(b, energy, acc64, warps, s);
    case 3: case 4: return launch_nt<4>(b, energy, acc64, warps, s);
    default: return launch_nt<8>(b, energy, acc64, warps, s);
  }
}

}  // namespace pb
