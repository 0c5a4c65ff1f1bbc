// Verlet neighbour list of one system.
//
// Replaces cudaParticleMD::makeNList (cudaParticleMD.cu:338-394: coordination
// numbers, CSR row pointers, then makeJlist_WithBlock_F4 over the cell list)
// and the list branch of cudaParticleMD::calcForce (cudaParticleMD.cu:41-44,
// calcF_IJpairWithList_F4 at kerneltemplate.hh:135-168).  The list holds, for
// every atom, the atoms within rc + thickness at the build; forces between
// builds use the list instead of the cell list, and the cell list is rebuilt
// only with the list, as testMD4n.cu:175-181 does.
//
// Layout.  Instead of CSR (a count pass, a scan and a fill pass), rows have a
// fixed capacity and are stored column-major: entry k of row s at
// idx[k * N + s], so the threads of a warp (consecutive rows) read one
// coalesced line per entry.  Row s belongs to the atom that sat in sorted slot
// s at the build, and entries are build-time slots too: every force call first
// copies the current positions into that order (rl), so a warp's atoms are
// neighbours of one another and the positions they gather sit in a few nearby
// lines, mostly shared through L1.  The build reports the longest row; the
// host grows the capacity and rebuilds when a row did not fit.
//
// Minimum image.  Each component of a pair difference is x_i - x_j, and when
// that exceeds half the box the coordinate above the box middle is moved down
// by L first, which is exact; the result is the minimum-image displacement
// without the rounding of a large intermediate.
//
// Staleness.  The force kernel compares every atom's position with its
// position at the build and raises kStatusStaleList when it moved more than
// half the skin: the list may then miss a pair inside the cutoff.
#include "md.cuh"

namespace pb {
namespace {

constexpr int kNlThreads = 256;

__device__ __forceinline__ float image_delta(float xi, float xj, float L, float hL) {
  const float d = xi - xj;
  if (d > hL) return (xi - L) - xj;
  if (d < -hL) return xi - (xj - L);
  return d;
}

__device__ __forceinline__ float round_image(float d, float L, float Linv) {
  return d - L * rintf(d * Linv);
}

// Row s of the list, built by one thread; returns its length (entries beyond
// the capacity are counted, not stored).  The three cells z - 1, z, z + 1 of a neighbour column
// are consecutive in sorted order and sorted by z, so each column is one
// range: a binary search finds its first atom inside the atom's z window,
// and the scan stops at the first atom above it.  The window half-width
// shrinks with the atom's distance in x and y from that column, a bound
// taken with a margin of 10^-3 cell edges (cell membership is decided in
// FP32).  The column's periodic image is applied as one shift.  A column
// whose z cells wrap around the box (z = 0 or nz - 1) is scanned cell by
// cell, with a shift per cell.  Candidates are visited in sorted order, so a
// row lists its atoms in the same order as a scan of the 27 cells.
__device__ uint32_t nlist_row(const NlistBufs &b, uint32_t s) {
  const SysDesc &S = b.sys[0];
  const Grid g = S.g;
  const int nx = g.n[0], ny = g.n[1], nz = g.n[2];
  const float Lx = g.L[0], Ly = g.L[1], Lz = g.L[2];
  const uint32_t i = b.pid[s];
  const float4 p = b.rs[s];
  const uint32_t kk = b.key[i] - S.cell0;
  const uint32_t rank = kk / (uint32_t)nz;
  const int z = (int)(kk - rank * (uint32_t)nz);
  const uint32_t xy = b.colxy[S.col0 + rank];
  const int d0 = (int)(xy / (uint32_t)ny), d1 = (int)(xy % (uint32_t)ny);
  // distances to the home cell's x and y faces, less the margin
  const float mx = 1e-3f * g.len[0], my = 1e-3f * g.len[1];
  const float xlo = g.lo[0] + (float)d0 * g.len[0], xhi = xlo + g.len[0];
  const float ylo = g.lo[1] + (float)d1 * g.len[1], yhi = ylo + g.len[1];
  const float ex_lo = fmaxf(p.x - xlo - mx, 0.f), ex_hi = fmaxf(xhi - p.x - mx, 0.f);
  const float ey_lo = fmaxf(p.y - ylo - my, 0.f), ey_hi = fmaxf(yhi - p.y - my, 0.f);
  const bool wraps = z == 0 || z == nz - 1;
  uint32_t n = 0;
  auto take = [&](uint32_t t, float qx, float qy, float qz, float sx, float sy, float sz) {
    const float dx = (qx + sx) - p.x, dy = (qy + sy) - p.y, dz = (qz + sz) - p.z;
    if (t != s && fmaf(dx, dx, fmaf(dy, dy, dz * dz)) < b.rl2) {
      if (n < b.cap) b.idx[(size_t)n * b.N + s] = t;
      ++n;
    }
  };
  for (int a = -1; a <= 1; ++a) {
    const float ex = a < 0 ? ex_lo : (a > 0 ? ex_hi : 0.f);
    const float sx = d0 + a < 0 ? -Lx : (d0 + a >= nx ? Lx : 0.f);
    for (int c = -1; c <= 1; ++c) {
      const float ey = c < 0 ? ey_lo : (c > 0 ? ey_hi : 0.f);
      const float rem = b.rl2 - fmaf(ex, ex, ey * ey);
      if (!(rem > 0.f)) continue;  // the whole column is out of range
      const float sy = d1 + c < 0 ? -Ly : (d1 + c >= ny ? Ly : 0.f);
      const int c0 = (d0 + a + nx) % nx, c1 = (d1 + c + ny) % ny;
      const uint32_t rk = b.colrank[S.col0 + (uint32_t)(c0 * ny + c1)];
      const uint32_t kb = S.cell0 + rk * (uint32_t)nz;
      if (wraps) {
        for (int e = -1; e <= 1; ++e) {
          const int ze = z + e;
          const float sz = ze < 0 ? -Lz : (ze >= nz ? Lz : 0.f);
          const uint32_t key2 = kb + (uint32_t)((ze + nz) % nz);
          const uint32_t t1 = b.start[key2 + 1];
          for (uint32_t t0 = b.start[key2]; t0 < t1; t0 += 4) {
            float4 q[4];  // four candidates per pass, their loads issued together
#pragma unroll
            for (int u = 0; u < 4; ++u) q[u] = b.rs[min(t0 + u, t1 - 1)];
#pragma unroll
            for (int u = 0; u < 4; ++u)
              if (t0 + u < t1) take(t0 + u, q[u].x, q[u].y, q[u].z, sx, sy, sz);
          }
        }
        continue;
      }
      const float dzw = sqrtf(rem) * 1.0001f;
      const float zlo = p.z - dzw, zhi = p.z + dzw;
      uint32_t lo = b.start[kb + (uint32_t)(z - 1)];
      uint32_t hi = b.start[kb + (uint32_t)(z + 2)];
      // first atom with z >= zlo
      uint32_t len = hi - lo;
      while (len > 0) {
        const uint32_t half = len >> 1;
        if (__ldg(&b.rs[lo + half].z) < zlo) {
          lo += half + 1;
          len -= half + 1;
        } else {
          len = half;
        }
      }
      bool past = false;
      for (uint32_t t0 = lo; t0 < hi && !past; t0 += 4) {
        float4 q[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) q[u] = b.rs[min(t0 + u, hi - 1)];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          past = past || t0 + u >= hi || q[u].z > zhi;
          if (!past) take(t0 + u, q[u].x, q[u].y, q[u].z, sx, sy, 0.f);
        }
      }
    }
  }
  b.cnt[s] = n;
  b.atom[s] = i;
  b.r0[s] = make_float4(p.x, p.y, p.z, 0.0f);
  if (n > b.cap) atomicOr(&b.status[0], kStatusNlistOverflow);
  return n;
}

__global__ void __launch_bounds__(kNlThreads) k_nlist_build(NlistBufs b) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  // the longest row goes to one counter: a maximum over the warp first, then
  // one atomic per warp (an atomic per row on one address serialises)
  const uint32_t n = s < b.N ? nlist_row(b, s) : 0u;
  const uint32_t wmax = __reduce_max_sync(0xffffffffu, n);
  if ((threadIdx.x & 31) == 0 && wmax > 0) atomicMax(b.maxcnt, wmax);
}

// Current positions in row order, so the pair loop gathers from build-time
// slots (type id bits in w, as in the sorted positions).
__global__ void __launch_bounds__(kNlThreads) k_nlist_gather(NlistBufs b) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= b.N) return;
  const uint32_t i = b.atom[s];
  const float4 p = b.r[i];
  b.rl[s] = make_float4(p.x, p.y, p.z, __int_as_float((int)b.type[i]));
}

template <int NT, bool ENERGY, typename Acc>
__global__ void __launch_bounds__(kNlThreads) k_nlist_force(NlistBufs b) {
  __shared__ float s2[NT * NT], e24[NT * NT], e4[NT * NT], rc2[NT * NT], ush[NT * NT];
  __shared__ double red[4 * 32];
  if (threadIdx.x < NT * NT) {
    const LJTable &T = b.lj[0];
    const int k = (threadIdx.x / NT) * T.nt + threadIdx.x % NT;
    s2[threadIdx.x] = T.s2[k];
    e24[threadIdx.x] = T.e24[k];
    e4[threadIdx.x] = T.e4[k];
    rc2[threadIdx.x] = T.rc2[k];
    ush[threadIdx.x] = T.ushift[k];
  }
  __syncthreads();
  const Grid g = b.sys[0].g;
  const float Lx = g.L[0], Ly = g.L[1], Lz = g.L[2];
  const float hx = 0.5f * Lx, hy = 0.5f * Ly, hz = 0.5f * Lz;
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  Acc pe = 0, pes = 0, vir = 0;
  uint32_t npairs = 0;
  if (s < b.N) {
    const uint32_t i = b.atom[s];
    const float4 p = b.rl[s];
    const int ti = NT == 1 ? 0 : __float_as_int(p.w);
    const uint32_t n = min(b.cnt[s], b.cap);
    Acc fx = 0, fy = 0, fz = 0;
    // four entries per pass: their row reads, then their position gathers, are
    // issued before any of them is used (memory-level parallelism)
    constexpr int kU = 4;
    for (uint32_t k0 = 0; k0 < n; k0 += kU) {
      uint32_t t[kU];
#pragma unroll
      for (int u = 0; u < kU; ++u)
        t[u] = k0 + u < n ? __ldg(&b.idx[(size_t)(k0 + u) * b.N + s]) : s;
      float4 q[kU];
#pragma unroll
      for (int u = 0; u < kU; ++u) q[u] = b.rl[t[u]];
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        const float dx = image_delta(p.x, q[u].x, Lx, hx);
        const float dy = image_delta(p.y, q[u].y, Ly, hy);
        const float dz = image_delta(p.z, q[u].z, Lz, hz);
        const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
        const int kk = NT == 1 ? 0 : ti * NT + __float_as_int(q[u].w);
        // padding entries point at the atom itself: r2 = 0, never counted
        if (r2 < rc2[kk] && r2 > 0.0f) {
          const float inv = rcp_approx(r2);
          const float sr2 = s2[kk] * inv;
          const float sr6 = sr2 * sr2 * sr2;
          const float f = e24[kk] * sr6 * fmaf(2.0f, sr6, -1.0f) * inv;
          fx += (Acc)(f * dx);
          fy += (Acc)(f * dy);
          fz += (Acc)(f * dz);
          if (ENERGY) {
            const float u2 = e4[kk] * sr6 * (sr6 - 1.0f);
            pe += (Acc)(0.5f * u2);
            pes += (Acc)(0.5f * (u2 - ush[kk]));
            vir += (Acc)(0.5f * f * r2);
            ++npairs;
          }
        }
      }
    }
    b.F[i] = make_float4((float)fx, (float)fy, (float)fz, 0.0f);
    // has the atom left the skin the list was built with?
    const float4 p0 = b.r0[s];
    const float ex = image_delta(p.x, p0.x, Lx, hx), ey = image_delta(p.y, p0.y, Ly, hy);
    const float ez = image_delta(p.z, p0.z, Lz, hz);
    if (fmaf(ex, ex, fmaf(ey, ey, ez * ez)) > 0.25f * b.skin * b.skin)
      atomicOr(&b.status[0], kStatusStaleList);
  }
  if (ENERGY) {
    double v[4] = {(double)pe, (double)pes, (double)vir, (double)npairs};
    block_sum<4>(v, red);
    if (threadIdx.x == 0)
      for (int k = 0; k < 4; ++k) b.partials[(size_t)blockIdx.x * 4 + k] = v[k];
  }
}

template <int NT>
cudaError_t launch_nt(const NlistBufs &b, bool energy, bool acc64, cudaStream_t s) {
  const uint32_t nb = nlist_blocks(b.N);
  k_nlist_gather<<<nb, kNlThreads, 0, s>>>(b);
  if (energy) {
    if (acc64) k_nlist_force<NT, true, double><<<nb, kNlThreads, 0, s>>>(b);
    else k_nlist_force<NT, true, float><<<nb, kNlThreads, 0, s>>>(b);
  } else {
    if (acc64) k_nlist_force<NT, false, double><<<nb, kNlThreads, 0, s>>>(b);
    else k_nlist_force<NT, false, float><<<nb, kNlThreads, 0, s>>>(b);
  }
  return cudaGetLastError();
}

}  // namespace

uint32_t nlist_blocks(uint32_t N) { return (N + kNlThreads - 1) / kNlThreads; }

cudaError_t launch_nlist_build(const NlistBufs &b, cudaStream_t s) {
  if (b.N == 0) return cudaSuccess;
  k_nlist_build<<<nlist_blocks(b.N), kNlThreads, 0, s>>>(b);
  return cudaGetLastError();
}

cudaError_t launch_nlist_force(const NlistBufs &b, int nt_max, bool energy, bool acc64,
                               cudaStream_t s) {
  if (b.N == 0) return cudaSuccess;
  switch (nt_max) {
    case 1: return launch_nt<1>(b, energy, acc64, s);
    case 2: return launch_nt<2>(b, energy, acc64, s);
    case 3: case 4: return launch_nt<4>(b, energy, acc64, s);
    default: return launch_nt<8>(b, energy, acc64, s);
  }
}

}  // namespace pb
