#include "plan.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>

namespace pb {

bool make_grid(const float cell6[6], float rmax, Grid &g, bool periodic) {
  for (int i = 0; i < 3; ++i) {
    const float c = cell6[2 * i + 1] - cell6[2 * i];
    const float q = c / rmax;
    if (periodic) {
      if (!(q >= 3.0f) || q > 1.0e6f) return false;
      g.n[i] = static_cast<int>(static_cast<uint32_t>(q));
      g.len[i] = c / static_cast<float>(static_cast<uint32_t>(g.n[i]));
    } else {
      if (!(q >= 2.0f) || q > 1.0e6f) return false;
      g.n[i] = static_cast<int>(static_cast<uint32_t>(q) + 1u);
      g.len[i] = rmax;
    }
    g.lo[i] = cell6[2 * i];
    g.L[i] = c;
  }
  g.periodic = periodic ? 1 : 0;
  const uint64_t nc = (uint64_t)g.n[0] * g.n[1] * g.n[2];
  if (nc >= 0xffffffffull) return false;
  g.ncells = (uint32_t)nc;
  return true;
}

static uint64_t spread_bits(uint32_t v) {
  uint64_t x = v;
  x = (x | (x << 16)) & 0x0000ffff0000ffffull;
  x = (x | (x << 8)) & 0x00ff00ff00ff00ffull;
  x = (x | (x << 4)) & 0x0f0f0f0f0f0f0f0full;
  x = (x | (x << 2)) & 0x3333333333333333ull;
  x = (x | (x << 1)) & 0x5555555555555555ull;
  return x;
}

void morton_columns(int nx, int ny, std::vector<uint32_t> &rank, std::vector<uint32_t> &xy) {
  const uint32_t nc = (uint32_t)nx * ny;
  std::vector<std::pair<uint64_t, uint32_t>> code(nc);
  for (int a = 0; a < nx; ++a)
    for (int b = 0; b < ny; ++b) {
      const uint32_t c = (uint32_t)a * ny + b;
      code[c] = {spread_bits((uint32_t)a) | (spread_bits((uint32_t)b) << 1), c};
    }
  std::sort(code.begin(), code.end());
  rank.assign(nc, 0);
  xy.assign(nc, 0);
  for (uint32_t k = 0; k < nc; ++k) {
    rank[code[k].second] = k;
    xy[k] = code[k].second;
  }
}

void neighbor_table(const Grid &g, std::vector<uint32_t> &out) {
  const long nx = g.n[0], ny = g.n[1], nz = g.n[2];
  out.assign((size_t)g.ncells * 27, 0);
  for (long i = 0; i < nx; ++i)
    for (long j = 0; j < ny; ++j)
      for (long k = 0; k < nz; ++k) {
        const size_t I = (size_t)(k + j * nz + i * nz * ny);
        int L = 0;
        for (int a = -1; a <= 1; ++a)
          for (int b = -1; b <= 1; ++b)
            for (int c = -1; c <= 1; ++c) {
              const bool inside = i + a >= 0 && i + a < nx && j + b >= 0 && j + b < ny &&
                                  k + c >= 0 && k + c < nz;
              const long i2 = (i + a + nx) % nx, j2 = (j + b + ny) % ny, k2 = (k + c + nz) % nz;
              out[I * 27 + L++] = g.periodic || inside ? (uint32_t)(k2 + j2 * nz + i2 * nz * ny)
                                                       : kNoCell;
            }
      }
}

// Environment overrides, read once per process.
static const char *env_once(int slot) {
  static const char *v[2] = {std::getenv("PB_FORCE_SEG"), std::getenv("PB_FORCE_CAP")};
  return v[slot];
}

int choose_segment(double atoms_per_cell, int nz, double scale, int nt, bool half) {
  // about 200 home atoms (25 clusters of 8) per force work item; PB_FORCE_SEG
  // overrides.  Shorter runs while the stage would not let two force CTAs
  // share an SM.
  const double apc = std::max(atoms_per_cell, 1.0);
  int seg = (int)std::lround(200.0 * scale / apc);
  if (const char *e = env_once(0)) seg = std::atoi(e);
  seg = std::max(1, std::min(seg, force_max_segment()));
  seg = std::min(seg, nz);
  // the kernel that runs sets the limit; the full-shell one also serves the
  // soft-core and relaxation forces, so it always has to fit
  while (seg > 1 && (force_smem_per_cta(choose_capacity(apc, seg), nt) > force_smem_limit() ||
                     (half && force_half_smem_per_cta(choose_capacity_half(apc, seg), nt) >
                                  112 * 1024)))
    --seg;
  return seg;
}

int choose_bucket_cap(double atoms_per_cell) {
  const double want = 2.0 * std::max(atoms_per_cell, 0.0) + 8.0;
  const int cap = ((int)std::ceil(want) + 7) & ~7;
  return std::max(32, std::min(cap, 1024));
}

int choose_tile_atoms(double atoms_per_cell) {
  const double want = 64.0 * 1.3 * std::max(atoms_per_cell, 0.0) + 64.0;
  const int n = ((int)std::ceil(want) + 31) & ~31;
  return std::max(256, std::min(n, 4096));
}

int choose_capacity(double atoms_per_cell, int seg) {
  const double expect = 9.0 * (seg + 2) * std::max(atoms_per_cell, 1.0);
  double factor = 1.15;  // headroom over the mean occupancy; PB_FORCE_CAP overrides
  if (const char *e = env_once(1)) factor = std::atof(e);
  const double cap = factor * expect + 128.0;
  // the largest launch shape (8 warps, 8 types) bounds every launch's memory
  static const double max_atoms = (double)force_max_capacity(8, kMaxTypes);
  return (int)std::min(cap, max_atoms);
}

int choose_capacity_half(double atoms_per_cell, int seg) {
  const double expect = 5.0 * (seg + 2) * std::max(atoms_per_cell, 1.0);
  double factor = 1.15;
  if (const char *e = env_once(1)) factor = std::atof(e);
  const double cap = factor * expect + 128.0;
  static const double max_atoms = (double)force_half_max_capacity(kMaxTypes);
  return (int)std::min(cap, max_atoms);
}

// z runs of one column: a top run of t <= nz/2 - 1 cells (its staged cells,
// from z0 - 1 up, then all lie at z >= L/2, where the force kernel's frame
// shift by -L is exact), the rest split evenly into runs of at most `seg`.
// Every column gets at least two runs, so no run touches both faces.
void append_items(uint32_t sys, const Grid &g, int seg, uint32_t cell0,
                  const std::vector<uint32_t> &rank, const std::vector<uint32_t> &xy,
                  std::vector<ForceItem> &items) {
  const uint32_t ncol = (uint32_t)g.n[0] * g.n[1];
  const int nx = g.n[0], ny = g.n[1], nz = g.n[2];
  // a column that fits one run is one item; otherwise a top run of at most
  // nz / 2 - 1 cells (its frame shift is exact) and runs of at most seg below
  const bool whole = nz <= seg;
  const int t = whole ? nz : std::max(1, std::min(seg, nz / 2 - 1));
  const int rest = nz - t;
  const int parts = whole ? 0 : std::max(1, (rest + seg - 1) / seg);
  for (uint32_t c = 0; c < ncol; ++c) {
    ForceItem it{};
    it.sys = sys;
    it.col = c;
    const int cx = (int)(xy[c] / (uint32_t)ny), cy = (int)(xy[c] % (uint32_t)ny);
    it.cx = (uint16_t)cx;
    it.cy = (uint16_t)cy;
    for (int k = 0; k < 9; ++k) {
      const int ax0 = cx + k / 3 - 1, ay0 = cy + k % 3 - 1;
      const int ax = (ax0 + nx) % nx, ay = (ay0 + ny) % ny;
      const bool inside = ax0 >= 0 && ax0 < nx && ay0 >= 0 && ay0 < ny;
      // an open box has no column past its faces
      it.kbase[k] = g.periodic || inside ? cell0 + rank[(size_t)ax * ny + ay] * (uint32_t)nz
                                         : kNoCell;
    }
    int z = 0;
    for (int p = 0; p < parts; ++p) {
      const int len = rest / parts + (p < rest % parts ? 1 : 0);
      it.z0 = (uint16_t)z;
      it.z1 = (uint16_t)(z + len);
      items.push_back(it);
      z += len;
    }
    it.z0 = (uint16_t)rest;
    it.z1 = (uint16_t)nz;
    items.push_back(it);
  }
}

}  // namespace pb
