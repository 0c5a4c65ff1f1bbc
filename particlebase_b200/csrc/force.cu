// Lennard-Jones pair forces over the cell list.
//
// Replaces cudaParticleMD::calcForce (cudaParticleMD.cu:24-69):
// calcF_IJpairWithBlock_F4<MDpairForce<potentialLJ>> on a (cells x 27) grid
// writing 27 partial-force planes tmp81N, followed by reduce27_F4
// (kerneltemplate.hh:229-294, kerneltemplate.hh:523-565, kernelinline.hh:86-96,
// kernelfuncs.cu:935-949).  The physics is the reference's: truncated,
// unshifted LJ, F_i = sum_{j != i, r < rc} 24 eps (s/r)^6 (2 (s/r)^6 - 1) / r^2
// (r_i - r_j) with the minimum image; all pairs inside rc of the 27-cell
// stencil contribute.  No 81 N scratch: each atom's force is summed in
// registers and written once.
//
// Work decomposition: one CTA per work item = (system, x-y column, run of z
// cells [z0, z1)).  The CTA stages the 3 x 3 neighbour columns over z cells
// [z0 - 1, z1] (with periodic z halo cells) into shared memory with 1-D bulk
// copies (cp.async.bulk, mbarrier completion; no multicast).  Each warp then
// takes 32 consecutive home atoms, one per lane, and sweeps the staged
// neighbours of the z cells the tile touches, every lane testing the same j
// (a shared-memory broadcast).
//
// Minimum image without rounding loss: positions are absolute FP32
// coordinates.  For a neighbour image below the box (j near the top face) the
// staged copy holds x_j - L, which is exact (Sterbenz) because x_j >= L/2; for
// an image above the box (j near the bottom face) the home coordinate is used
// as x_i - L instead, exact for the same reason.  Every difference x_i - x_j is
// then taken between numbers of similar magnitude, so the FP32 displacement is
// as accurate as the inputs allow even in a 190-sigma box.
#include "md.cuh"
#include "tma.cuh"

namespace pb {
namespace {

constexpr int kMaxSeg = 96;  // longest z run of one work item (cells)

template <int NT>
struct LJLocal {
  float s2[NT * NT], e24[NT * NT], e4[NT * NT], rc2[NT * NT], ush[NT * NT];
};

template <int NT, bool ENERGY, bool SELF, bool JSHIFT, typename Acc>
__device__ __forceinline__ void pair_range(const float4 *__restrict__ P, uint32_t jb,
                                           uint32_t je, float xi, float yi, float zi, int ti,
                                           float jsx, float jsy, float jsz, uint32_t self,
                                           const LJLocal<NT> &lj, Acc &fx, Acc &fy, Acc &fz,
                                           Acc &pe, Acc &pes, Acc &vir, uint32_t &npair) {
#pragma unroll 4
  for (uint32_t j = jb; j < je; ++j) {
    const float4 q = P[j];
    const float xj = JSHIFT ? q.x - jsx : q.x;
    const float yj = JSHIFT ? q.y - jsy : q.y;
    const float zj = JSHIFT ? q.z - jsz : q.z;
    const float dx = xi - xj, dy = yi - yj, dz = zi - zj;
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    const int k = NT == 1 ? 0 : ti * NT + __float_as_int(q.w);
    bool in = r2 < lj.rc2[k];
    if (SELF) in = in && (j != self);
    if (in) {
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
        ++npair;
      }
    }
  }
}

struct Stage {
  // staged index of the first atom of staged z cell k of column c (k = 0 is
  // image cell z0 - 1, k = nseg + 1 is image cell z1); entry nseg + 2 is the end
  uint32_t off[9][kMaxSeg + 3];
  uint32_t key_first[9];  // packed key of image cell z0 - 1 .. (used in global mode)
  int wx[9], wy[9];       // column wrap: -1 image below, +1 image above, 0 none
  uint64_t bar;
  uint32_t total;
  uint32_t home_g0;       // global sorted index of the first home atom
  int overflow;
};

template <int NT, bool ENERGY, typename Acc>
__global__ void __launch_bounds__(128) k_force(ForceBufs b) {
  extern __shared__ float4 sp[];
  __shared__ Stage st;
  __shared__ LJLocal<NT> ljs;
  __shared__ double red[4 * 32];

  const ForceItem it = b.items[blockIdx.x];
  const SysDesc &S = b.sys[it.sys];
  const Grid g = S.g;
  const int nx = g.n[0], ny = g.n[1], nz = g.n[2];
  const int z0 = it.z0, z1 = it.z1, nseg = z1 - z0;
  const uint32_t cxy = b.colxy[S.col0 + it.col];
  const int cx = (int)(cxy / (uint32_t)ny), cy = (int)(cxy % (uint32_t)ny);

  if (threadIdx.x < NT * NT) {
    const LJTable &T = b.lj[S.lj];
    const int a = threadIdx.x / NT, c = threadIdx.x % NT;
    const int k = a * T.nt + c;
    ljs.s2[threadIdx.x] = T.s2[k];
    ljs.e24[threadIdx.x] = T.e24[k];
    ljs.e4[threadIdx.x] = T.e4[k];
    ljs.rc2[threadIdx.x] = T.rc2[k];
    ljs.ush[threadIdx.x] = T.ushift[k];
  }
  // Cell counts of the 9 columns x (nseg + 2) staged cells.
  if (threadIdx.x < 9) {
    const int c = threadIdx.x;
    const int dx = c / 3 - 1, dy = c % 3 - 1;
    int ax = cx + dx, ay = cy + dy;
    st.wx[c] = ax < 0 ? -1 : (ax >= nx ? 1 : 0);
    st.wy[c] = ay < 0 ? -1 : (ay >= ny ? 1 : 0);
    ax = (ax + nx) % nx;
    ay = (ay + ny) % ny;
    const uint32_t rank = b.colrank[S.col0 + ax * ny + ay];
    const uint32_t kbase = S.cell0 + rank * (uint32_t)nz;
    st.key_first[c] = kbase;
    uint32_t acc = 0;
    for (int k = 0; k <= nseg + 1; ++k) {
      const int zc = (z0 - 1 + k + nz) % nz;
      st.off[c][k] = acc;
      acc += b.start[kbase + zc + 1] - b.start[kbase + zc];
    }
    st.off[c][nseg + 2] = acc;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t tot = 0;
    for (int c = 0; c < 9; ++c) {
      const uint32_t n = st.off[c][nseg + 2];
      for (int k = 0; k <= nseg + 2; ++k) st.off[c][k] += tot;
      tot += n;
    }
    st.total = tot;
    st.overflow = tot > (uint32_t)b.cap;
    st.home_g0 = b.start[st.key_first[4] + z0];
    if (!st.overflow && tot > 0) {
      mbar_init(&st.bar, 1);
      mbar_fence_init();
    }
  }
  __syncthreads();
  const bool overflow = st.overflow;
  if (!overflow && st.total > 0) {
    if (threadIdx.x == 0) {
      mbar_arrive_expect_tx(&st.bar, st.total * 16u);
      for (int c = 0; c < 9; ++c) {
        const uint32_t kb = st.key_first[c];
        // below halo (image z0 - 1), main run, above halo (image z1)
        int k = 0;
        while (k <= nseg + 1) {
          const int zc = (z0 - 1 + k + nz) % nz;
          int kend = k;  // extend while the next staged cell is the next key
          while (kend + 1 <= nseg + 1 && ((z0 - 1 + kend + 1 + nz) % nz) == zc + (kend + 1 - k)) ++kend;
          const uint32_t g0 = b.start[kb + zc];
          const uint32_t g1 = b.start[kb + zc + (kend - k) + 1];
          if (g1 > g0) bulk_g2s(&sp[st.off[c][k]], &b.rs[g0], (g1 - g0) * 16u, &st.bar);
          k = kend + 1;
        }
      }
    }
    const bool ok = mbar_wait_bounded(&st.bar, 0);
    if (__syncthreads_or(!ok)) {
      if (threadIdx.x == 0) atomicOr(b.status, kStatusWaitTimeout);
      return;
    }
    // Images below the box: x - L (exact, x near the top face).
    for (int c = 0; c < 9; ++c) {
      const bool sx = st.wx[c] < 0, sy = st.wy[c] < 0;
      if (sx || sy) {
        for (uint32_t q = st.off[c][0] + threadIdx.x; q < st.off[c][nseg + 2]; q += blockDim.x) {
          if (sx) sp[q].x -= g.L[0];
          if (sy) sp[q].y -= g.L[1];
        }
      }
      if (z0 == 0) {
        for (uint32_t q = st.off[c][0] + threadIdx.x; q < st.off[c][1]; q += blockDim.x)
          sp[q].z -= g.L[2];
      }
    }
    __syncthreads();
  } else if (overflow && threadIdx.x == 0) {
    atomicOr(b.status, kStatusSmemOverflow);
  }

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const uint32_t hbeg = st.off[4][1], hend = st.off[4][nseg + 1];
  const uint32_t H = hend - hbeg;
  Acc pe = 0, pes = 0, vir = 0;
  uint32_t npairs = 0;
  for (uint32_t t = warp; t * 32 < H; t += nwarps) {
    const uint32_t h = t * 32 + lane;
    const bool valid = h < H;
    const uint32_t hs = hbeg + (valid ? h : H - 1);  // staged index of the home atom
    // staged z cell of the home atom: largest k in [1, nseg] with off[4][k] <= hs
    int lo = 1, hi = nseg;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (st.off[4][mid] <= hs) lo = mid; else hi = mid - 1;
    }
    const int kh = lo;
    const int kmin = __reduce_min_sync(0xffffffffu, kh);
    const int kmax = __reduce_max_sync(0xffffffffu, kh);
    const uint32_t gh = st.home_g0 + (hs - hbeg);
    const float4 pi = overflow ? b.rs[gh] : sp[hs];
    const int ti = NT == 1 ? 0 : __float_as_int(pi.w);
    Acc fx = 0, fy = 0, fz = 0, tpe = 0, tpes = 0, tvir = 0;
    uint32_t tpair = 0;
    for (int c = 0; c < 9; ++c) {
      const float hx = st.wx[c] > 0 ? g.L[0] : 0.0f;
      const float hy = st.wy[c] > 0 ? g.L[1] : 0.0f;
      const float xi = pi.x - hx, yi = pi.y - hy;
      const int klast = kmax + 1;
      const bool above = (z1 == nz) && (klast == nseg + 1);
      if (!overflow) {
        const uint32_t jb = st.off[c][kmin - 1];
        const uint32_t je = st.off[c][above ? nseg + 1 : klast + 1];
        if (c == 4)
          pair_range<NT, ENERGY, true, false, Acc>(sp, jb, je, xi, yi, pi.z, ti, 0, 0, 0, hs,
                                                   ljs, fx, fy, fz, tpe, tpes, tvir, tpair);
        else
          pair_range<NT, ENERGY, false, false, Acc>(sp, jb, je, xi, yi, pi.z, ti, 0, 0, 0, 0,
                                                    ljs, fx, fy, fz, tpe, tpes, tvir, tpair);
        if (above) {
          const uint32_t ab = st.off[c][nseg + 1], ae = st.off[c][nseg + 2];
          const float zi = pi.z - g.L[2];
          if (c == 4)
            pair_range<NT, ENERGY, true, false, Acc>(sp, ab, ae, xi, yi, zi, ti, 0, 0, 0, hs,
                                                     ljs, fx, fy, fz, tpe, tpes, tvir, tpair);
          else
            pair_range<NT, ENERGY, false, false, Acc>(sp, ab, ae, xi, yi, zi, ti, 0, 0, 0, 0,
                                                      ljs, fx, fy, fz, tpe, tpes, tvir, tpair);
        }
      } else {
        // Global-memory fallback: walk the window cell by cell.
        const float jsx = st.wx[c] < 0 ? g.L[0] : 0.0f;
        const float jsy = st.wy[c] < 0 ? g.L[1] : 0.0f;
        for (int k = kmin - 1; k <= klast; ++k) {
          const int u = z0 - 1 + k;  // image z cell
          const int zc = (u + nz) % nz;
          const uint32_t key = st.key_first[c] + zc;
          const uint32_t jb = b.start[key], je = b.start[key + 1];
          const float jsz = u < 0 ? g.L[2] : 0.0f;
          const float zi = u >= nz ? pi.z - g.L[2] : pi.z;
          if (c == 4)
            pair_range<NT, ENERGY, true, true, Acc>(b.rs, jb, je, xi, yi, zi, ti, jsx, jsy, jsz,
                                                    gh, ljs, fx, fy, fz, tpe, tpes, tvir, tpair);
          else
            pair_range<NT, ENERGY, false, true, Acc>(b.rs, jb, je, xi, yi, zi, ti, jsx, jsy,
                                                     jsz, 0, ljs, fx, fy, fz, tpe, tpes, tvir, tpair);
        }
      }
    }
    if (valid) {  // padded lanes repeat the last home atom and write nothing
      const uint32_t p = b.pid[gh];
      b.F[p] = make_float4((float)fx, (float)fy, (float)fz, 0.0f);
      pe += tpe;
      pes += tpes;
      vir += tvir;
      npairs += tpair;
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

template <int NT, bool E, typename Acc>
cudaError_t launch_t(const ForceBufs &b, int threads, cudaStream_t s) {
  const size_t smem = (size_t)b.cap * sizeof(float4);
  auto kern = k_force<NT, E, Acc>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  kern<<<b.nitems, threads, smem, s>>>(b);
  return cudaGetLastError();
}

template <int NT>
cudaError_t launch_nt(const ForceBufs &b, bool energy, bool acc64, int threads, cudaStream_t s) {
  if (energy) {
    return acc64 ? launch_t<NT, true, double>(b, threads, s) : launch_t<NT, true, float>(b, threads, s);
  }
  return acc64 ? launch_t<NT, false, double>(b, threads, s) : launch_t<NT, false, float>(b, threads, s);
}

}  // namespace

int force_max_segment() { return kMaxSeg; }

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
