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
// Compute (shared-memory path).  Cells are sorted by z and atoms within a
// cell by z, so every staged column is one z-sorted array.  A warp takes a
// cluster of 8 consecutive home atoms (lane & 7) and splits the candidates 4
// ways (lane >> 3).  For each of the 9 columns it binary-searches the z window
// [z_min - rc, z_max + rc] of the cluster, then
//   phase 1  tests r^2 < rc^2 for its share of the window and appends the
//            hits to a per-lane index list in shared memory (no divergent
//            force code);
//   phase 2  evaluates the LJ force for the listed pairs.
// The 4 partial sums of an atom are combined with two warp shuffles.
// A CTA whose stage would exceed its shared-memory capacity computes from
// global memory instead (slower, same result) and raises a status bit.
#include "md.cuh"
#include "tma.cuh"

namespace pb {
namespace {

constexpr int kMaxSeg = 40;     // longest z run of one work item (cells)
constexpr int kDefaultWarps = 8;
constexpr int kListLen = 32;    // per-lane pair list entries before a flush

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
  // staged index of the first atom of staged z cell k of column c (k = 0 is
  // image cell z0 - 1, k = nseg + 1 is image cell z1); entry nseg + 2 is the end
  uint32_t off[9][kMaxSeg + 3];
  uint32_t kbase[9];   // packed key of z cell 0 of each column
  float sx[9], sy[9];  // frame shift of each column (0 or L)
  float sz_lo, sz_mid, sz_hi;  // frame shift of staged cell 0, 1..nseg, nseg + 1
  uint64_t bar;
  uint32_t total;
  uint32_t home_g0;    // global sorted index of the first home atom
  int overflow;
  int shifted;         // any nonzero frame shift in this CTA
};

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

__device__ __forceinline__ uint32_t lower_bound_z(const float4 *sp, uint32_t lo, uint32_t hi,
                                                  float key) {
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (sp[mid].z < key) lo = mid + 1; else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ uint32_t upper_bound_z(const float4 *sp, uint32_t lo, uint32_t hi,
                                                  float key) {
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (sp[mid].z <= key) lo = mid + 1; else hi = mid;
  }
  return lo;
}

template <int NT, bool ENERGY, typename Acc, int MODE>
__device__ __forceinline__ void flush_list(const float4 *sp, const uint16_t *list, uint32_t cnt,
                                           int lane, float4 pi, int ti, const LJLocal<NT> &lj,
                                           PairAcc<NT, ENERGY, Acc, MODE> &a) {
  if constexpr (NT == 1) {
    LJLocal<1> r;  // one type: parameters in registers
    r.s2[0] = lj.s2[0];
    r.e24[0] = lj.e24[0];
    r.e4[0] = lj.e4[0];
    r.rc2[0] = lj.rc2[0];
    r.ush[0] = lj.ush[0];
    r.sc_rc = lj.sc_rc;
    r.sc_f0 = lj.sc_f0;
    for (uint32_t k = 0; k < cnt; ++k) {
      const float4 q = sp[list[k * 32 + lane]];
      const float dx = pi.x - q.x, dy = pi.y - q.y, dz = pi.z - q.z;
      const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
      a.add(r, 0, dx, dy, dz, r2);
    }
    return;
  }
  for (uint32_t k = 0; k < cnt; ++k) {
    const float4 q = sp[list[k * 32 + lane]];
    const float dx = pi.x - q.x, dy = pi.y - q.y, dz = pi.z - q.z;
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    const int kk = NT == 1 ? 0 : ti * NT + __float_as_int(q.w);
    a.add(lj, kk, dx, dy, dz, r2);
  }
}

template <int NT, bool ENERGY, typename Acc, int kWarps, int MODE>
__global__ void __launch_bounds__(kWarps * 32, 32 / kWarps) k_force(ForceBufs b) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint16_t *lists = reinterpret_cast<uint16_t *>(smem_raw);                  // kWarps*kListLen*32
  float4 *sp = reinterpret_cast<float4 *>(smem_raw + kWarps * kListLen * 32 * 2);
  __shared__ Stage st;
  __shared__ LJLocal<NT> ljs;
  __shared__ uint32_t cnt_cell[9][kMaxSeg + 3];
  __shared__ uint32_t gstart[9][kMaxSeg + 3];
  __shared__ double red[4 * 32];

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

  if (threadIdx.x < NT * NT) {
    const LJTable &T = b.lj[S.lj];
    const int a = threadIdx.x / NT, c = threadIdx.x % NT;
    const int k = a * T.nt + c;
    ljs.s2[threadIdx.x] = T.s2[k];
    ljs.e24[threadIdx.x] = T.e24[k];
    ljs.e4[threadIdx.x] = T.e4[k];
    ljs.rc2[threadIdx.x] =
        MODE == kModeSoftCore ? fminf(T.rc2[k], b.sc_rc * b.sc_rc) : T.rc2[k];
    ljs.ush[threadIdx.x] = T.ushift[k];
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
  if (threadIdx.x < 32) {
    // exclusive prefix over (column, cell), column-major
    uint32_t run = 0;
    for (int c = 0; c < 9; ++c) {
      for (int base = 0; base < ncell; base += 32) {
        const int k = base + (int)threadIdx.x;
        const uint32_t v = k < ncell ? cnt_cell[c][k] : 0u;
        uint32_t incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
          if ((int)threadIdx.x >= o) incl += t;
        }
        if (k < ncell) st.off[c][k] = run + incl - v;
        run += __shfl_sync(0xffffffffu, incl, 31);
      }
      if (threadIdx.x == 0) st.off[c][ncell] = run;
    }
    if (threadIdx.x == 0) {
      st.total = run;
      st.overflow = run > S.cap;  // the system's own capacity: same path alone or batched
      st.home_g0 = gstart[4][1];
      bool sh = st.sz_lo != 0.f || st.sz_mid != 0.f || st.sz_hi != 0.f;
      for (int c = 0; c < 9; ++c) sh = sh || st.sx[c] != 0.f || st.sy[c] != 0.f;
      st.shifted = sh;
      if (!st.overflow && run > 0) {
        mbar_init(&st.bar, 9);
        mbar_fence_init();
      }
    }
  }
  __syncthreads();
  const bool overflow = st.overflow;
  if (!overflow && st.total > 0) {
    if (threadIdx.x < 9) {
      // column c: up to three contiguous runs (below halo, main, above halo)
      const int c = threadIdx.x;
      mbar_arrive_expect_tx(&st.bar, (st.off[c][ncell] - st.off[c][0]) * 16u);
      int k = 0;
      while (k < ncell) {
        const int zc = (z0 - 1 + k + nz) % nz;
        int kend = k;
        while (kend + 1 < ncell && ((z0 - 1 + kend + 1 + nz) % nz) == zc + (kend + 1 - k)) ++kend;
        const uint32_t g0 = gstart[c][k];
        const uint32_t g1 = gstart[c][kend] + cnt_cell[c][kend];
        if (g1 > g0) bulk_g2s(&sp[st.off[c][k]], &b.rs[g0], (g1 - g0) * 16u, &st.bar);
        k = kend + 1;
      }
    }
    const bool ok = mbar_wait_bounded(&st.bar, 0);
    if (__syncthreads_or(!ok)) {
      // give the copies in flight a second bounded wait before the CTA leaves
      if (threadIdx.x == 0) atomicOr(&b.status[it.sys], kStatusWaitTimeout);
      mbar_wait_bounded(&st.bar, 0);
      return;
    }
    if (st.shifted) {
      for (int c = 0; c < 9; ++c) {
        const float sx = st.sx[c], sy = st.sy[c];
        for (uint32_t q = st.off[c][0] + threadIdx.x; q < st.off[c][ncell]; q += blockDim.x) {
          const float sz = q < st.off[c][1] ? st.sz_lo
                                            : (q < st.off[c][nseg + 1] ? st.sz_mid : st.sz_hi);
          float4 p = sp[q];
          p.x -= sx;
          p.y -= sy;
          p.z -= sz;
          sp[q] = p;
        }
      }
      __syncthreads();
    }
  } else if (overflow && threadIdx.x == 0) {
    atomicOr(&b.status[it.sys], kStatusSmemOverflow);
  }

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t hbeg = st.off[4][1], hend = st.off[4][nseg + 1];
  const uint32_t H = hend - hbeg;
  Acc pe = 0, pes = 0, vir = 0;
  uint32_t npairs = 0;

  if (!overflow) {
    uint16_t *mylist = lists + warp * kListLen * 32;
    const int il = lane & 7, q = lane >> 3;
    float rcmax2 = 0.f;
    for (int k = 0; k < NT * NT; ++k) rcmax2 = fmaxf(rcmax2, ljs.rc2[k]);
    const float rcw = sqrtf(rcmax2) * 1.00001f + 1e-5f;
    const uint32_t nclus = (H + 7) / 8;
    for (uint32_t cl = warp; cl < nclus; cl += kWarps) {
      const uint32_t h = cl * 8 + il;
      const bool valid = h < H;
      const uint32_t hs = hbeg + (valid ? h : H - 1);
      const float4 pi = sp[hs];
      const float2 pxy = make_float2(pi.x, pi.y);
      const float2 m1 = make_float2(-1.0f, -1.0f);
      const int ti = NT == 1 ? 0 : __float_as_int(pi.w);
      // cutoff^2 of this lane's pairs; a padded lane gets -1 and never appends
      float rc2_1 = NT == 1 ? ljs.rc2[0] : 0.f;
      if (!valid) rc2_1 = -1.0f;
      const float zmin = sp[hbeg + cl * 8].z;
      const float zmax = sp[hbeg + min(cl * 8 + 7, H - 1)].z;
      // lanes 0..8: lower bound of column `lane`; lanes 16..24: upper bound
      uint32_t bound = 0;
      {
        const int c = lane & 15;
        if (c < 9) {
          const uint32_t lo = st.off[c][0], hi = st.off[c][ncell];
          bound = lane < 16 ? lower_bound_z(sp, lo, hi, zmin - rcw)
                            : upper_bound_z(sp, lo, hi, zmax + rcw);
        }
      }
      PairAcc<NT, ENERGY, Acc, MODE> acc;
      uint32_t cnt = 0;
      for (int c = 0; c < 9; ++c) {
        const uint32_t jlo = __shfl_sync(0xffffffffu, bound, c);
        const uint32_t jhi = __shfl_sync(0xffffffffu, bound, 16 + c);
        // chunks of at most 4 * kListLen candidates, so a lane appends at most
        // kListLen entries between flushes
        for (uint32_t jb = jlo; jb < jhi; jb += 4 * kListLen) {
          const uint32_t je = min(jhi, jb + 4 * kListLen);
          const uint32_t need = (je - jb + 3) >> 2;
          if (__reduce_max_sync(0xffffffffu, cnt) + need > (uint32_t)kListLen) {
            flush_list<NT, ENERGY, Acc, MODE>(sp, mylist, cnt, lane, pi, ti, ljs, acc);
            cnt = 0;
            __syncwarp();
          }
          uint16_t *out = mylist + cnt * 32 + lane;
          // this lane's candidates: j = jb + q + 4 t, t < n
          const int n = (int)je - (int)jb - q > 0 ? ((int)je - (int)jb - q + 3) >> 2 : 0;
          const float4 *pj = sp + jb + q;
          uint32_t j = jb + q;
          if (c == 4) {
#pragma unroll 4
            for (int t = 0; t < n; ++t, j += 4) {
              const float4 qj = pj[4 * t];
              // x and y differences as one packed FP32x2 pair (p - q exactly, FMA by -1)
              const float2 dxy = __ffma2_rn(make_float2(qj.x, qj.y), m1, pxy);
              const float2 sq = __fmul2_rn(dxy, dxy);
              const float dz = pi.z - qj.z;
              const float r2 = fmaf(dz, dz, sq.x + sq.y);
              const float rc2 = NT == 1 ? rc2_1 : (valid ? ljs.rc2[ti * NT + __float_as_int(qj.w)] : -1.f);
              // the store is in bounds whether or not it is kept: the chunk
              // check above leaves room for every candidate of this chunk
              *out = (uint16_t)j;
              out += (r2 < rc2 && j != hs) ? 32 : 0;
            }
          } else {
#pragma unroll 4
            for (int t = 0; t < n; ++t, j += 4) {
              const float4 qj = pj[4 * t];
              // x and y differences as one packed FP32x2 pair (p - q exactly, FMA by -1)
              const float2 dxy = __ffma2_rn(make_float2(qj.x, qj.y), m1, pxy);
              const float2 sq = __fmul2_rn(dxy, dxy);
              const float dz = pi.z - qj.z;
              const float r2 = fmaf(dz, dz, sq.x + sq.y);
              const float rc2 = NT == 1 ? rc2_1 : (valid ? ljs.rc2[ti * NT + __float_as_int(qj.w)] : -1.f);
              *out = (uint16_t)j;
              out += (r2 < rc2) ? 32 : 0;
            }
          }
          cnt = (uint32_t)(out - (mylist + lane)) >> 5;
        }
      }
      flush_list<NT, ENERGY, Acc, MODE>(sp, mylist, cnt, lane, pi, ti, ljs, acc);
      __syncwarp();
      // combine the 4 partial sums of each home atom (lanes il, il+8, il+16, il+24)
#pragma unroll
      for (int o = 8; o < 32; o <<= 1) {
        acc.fx += __shfl_xor_sync(0xffffffffu, acc.fx, o);
        acc.fy += __shfl_xor_sync(0xffffffffu, acc.fy, o);
        acc.fz += __shfl_xor_sync(0xffffffffu, acc.fz, o);
      }
      if (valid && q == 0) {
        const uint32_t gh = st.home_g0 + (hs - hbeg);
        b.F[b.pid[gh]] = make_float4((float)acc.fx, (float)acc.fy, (float)acc.fz, 0.0f);
      }
      if (ENERGY) {
        pe += acc.pe;
        pes += acc.pes;
        vir += acc.vir;
        npairs += acc.n;
      }
    }
  } else {
    // Global-memory path: 32 consecutive home atoms per warp, one per lane.
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
            global_range<NT, ENERGY, true, Acc, MODE>(b.rs, b.start[key], b.start[key + 1], xi, yi, zi,
                                                ti, st.sx[c], st.sy[c], sz, gh, ljs, acc);
          else
            global_range<NT, ENERGY, false, Acc, MODE>(b.rs, b.start[key], b.start[key + 1], xi, yi,
                                                 zi, ti, st.sx[c], st.sy[c], sz, 0, ljs, acc);
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
  const size_t smem = (size_t)W * kListLen * 32 * 2 + (size_t)b.cap * sizeof(float4);
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
