// FP64 CPU restatement of the reference's Lennard-Jones cell-list MD step.
//
// TEST INFRASTRUCTURE ONLY.  This is the oracle the CUDA path is checked
// against; it is loaded by tests/, by bench.py's CPU-baseline and reference
// arms and by __graft_entry__.smoke(), never by the product library.
// It is itself pinned against the reference's own kernels, compiled for the
// CPU into oracle/_ref (ref_harness.cpp), and against golden vectors made from
// those kernels (tests/golden/make_golden.py).
//
// Every function cites the reference code it restates (paths relative to the
// particlelover/ParticleBase checkout).  Arithmetic is FP64 except where the
// reference result depends on FP32 rounding that must be reproduced bit for
// bit: the cell grid (cudaCutoffBlock.cu:97-101) and the per-atom cell hash
// (kernelfuncs.cu:807-841), which are computed exactly as the reference does
// in IEEE single precision.
//
// Extensions beyond the reference (labelled where they appear): per-type-pair
// cutoffs, the shifted-energy bookkeeping used for drift, the closed-form
// Gaussian solve used as a cross-check, and steepest-descent relaxation.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>
#include <omp.h>

namespace {

constexpr int kMaxTypes = 8;

struct Grid {
  uint32_t n[3];
  float len[3];
  float lo[3];
  uint32_t ncells;
};

// cudaCutoffBlock::setupCutoffBlock (cudaCutoffBlock.cu:97-113), all in FP32.
// Periodic: blocknum = (uint32)(c / rmax), blocklen = c / (float)blocknum.
// Open: blocklen = rmax, blocknum = (uint32)(c / rmax) + 1.
int make_grid(const float *cell6, float rmax, Grid &g, int periodic = 1) {
  for (int i = 0; i < 3; ++i) {
    const float c = cell6[2 * i + 1] - cell6[2 * i];
    const float q = c / rmax;
    if (periodic) {
      g.n[i] = static_cast<uint32_t>(q);
      g.len[i] = c / static_cast<float>(g.n[i]);
    } else {
      g.n[i] = static_cast<uint32_t>(q) + 1u;
      g.len[i] = rmax;
    }
    if (!(q >= 0.0f) || g.n[i] <= 2) return -1;  // reference asserts blocknum > 2
    g.lo[i] = cell6[2 * i];
  }
  g.ncells = g.n[0] * g.n[1] * g.n[2];
  return 0;
}

// Device float->uint32 conversion as used by calcBID_F4: truncation toward
// zero, saturating (negative values and NaN become 0, too-large values become
// UINT_MAX).  This is the PTX cvt.rzi.u32.f32 rule.
inline uint32_t f2u_sat(float x) {
  if (!(x > 0.0f)) return 0u;
  if (x >= 4294967296.0f) return 0xffffffffu;
  return static_cast<uint32_t>(x);
}

// calcBID_F4 (kernelfuncs.cu:807-841): per-dimension index in FP32 with the
// two clamps (d == n -> n-1, d > n -> 0); id = d2 + d1*nz + d0*nz*ny.
inline uint32_t cell_of(const Grid &g, float x, float y, float z) {
  const float v[3] = {x, y, z};
  uint32_t d[3];
  for (int k = 0; k < 3; ++k) {
    uint32_t q = f2u_sat((v[k] - g.lo[k]) / g.len[k]);
    if (q == g.n[k]) {
      q = g.n[k] - 1;
    } else if (q > g.n[k]) {
      q = 0;
    }
    d[k] = q;
  }
  return d[2] + d[1] * g.n[2] + d[0] * g.n[2] * g.n[1];
}

// calc_BlockNeighbor (cudaCutoffBlock.cu:17-65), w = 1, 27 entries per cell,
// order: x offset outermost, z offset innermost, each over {-1, 0, +1}.
void neighbor_table(const Grid &g, int periodic, uint32_t *out) {
  const long nx = g.n[0], ny = g.n[1], nz = g.n[2];
#pragma omp parallel for schedule(static)
  for (long i = 0; i < nx; ++i)
    for (long j = 0; j < ny; ++j)
      for (long k = 0; k < nz; ++k) {
        const uint64_t I = (uint64_t)(k + j * nz + i * nz * ny);
        int L = 0;
        for (int a = -1; a <= 1; ++a)
          for (int b = -1; b <= 1; ++b)
            for (int c = -1; c <= 1; ++c) {
              long i2 = i + a, j2 = j + b, k2 = k + c;
              const bool inside = i2 >= 0 && i2 < nx && j2 >= 0 && j2 < ny && k2 >= 0 && k2 < nz;
              i2 = (i2 + nx) % nx;
              j2 = (j2 + ny) % ny;
              k2 = (k2 + nz) % nz;
              uint32_t J = 0xffffffffu;
              if (periodic || inside) J = (uint32_t)(k2 + j2 * nz + i2 * nz * ny);
              out[I * 27 + L++] = J;
            }
      }
}

// Counting sort of atoms by cell id.  Replaces the reference's racy
// single-CTA sort (sortByBID_M1 + sortByBID + makeBindex,
// kernelfuncs.cu:844-932): the per-cell member sets and counts are the same;
// the within-cell order, history-dependent in the reference, is made
// canonical: ascending FP32 z coordinate, ties by ascending particle id
// (NaN coordinates last).
// `z` may be null, giving ascending particle id.
void cell_list(const uint32_t *cid, const float *z, uint32_t N, uint32_t ncells,
               uint32_t *start, uint32_t *members) {
  std::vector<uint32_t> cnt(ncells + 1, 0);
  for (uint32_t i = 0; i < N; ++i) cnt[cid[i] + 1]++;
  for (uint32_t c = 0; c < ncells; ++c) cnt[c + 1] += cnt[c];
  std::memcpy(start, cnt.data(), sizeof(uint32_t) * (ncells + 1));
  for (uint32_t i = 0; i < N; ++i) members[cnt[cid[i]]++] = i;
  if (z) {
    // NaN coordinates sort after every number (ties by id), so the order is
    // a strict total order whatever the input
    auto key = [z](uint32_t a) { return std::isnan(z[a]) ? 1 : 0; };
    for (uint32_t c = 0; c < ncells; ++c)
      std::sort(members + start[c], members + start[c + 1], [z, key](uint32_t a, uint32_t b) {
        const int na = key(a), nb = key(b);
        if (na != nb) return na < nb;
        return (!na && z[a] < z[b]) || ((na || z[a] == z[b]) && a < b);
      });
  }
}

struct LJTable {
  int ntypes = 1;
  double s2[kMaxTypes * kMaxTypes];
  double e24[kMaxTypes * kMaxTypes];
  double e4[kMaxTypes * kMaxTypes];
  double rc2[kMaxTypes * kMaxTypes];
  double ushift[kMaxTypes * kMaxTypes];  // U(rc), for the shifted energy
};

// _setLJparams (kernelinline.hh:120-134) stores {sigma^2, 24 eps} per pair.
// The reference has one global cutoff rmax2 (kerneltemplate.hh:533); the
// table also carries a cutoff per pair (extension for Kob-Andersen mixtures).
void make_table(const double *lj, int ntypes, LJTable &t) {
  t.ntypes = ntypes;
  for (int a = 0; a < ntypes; ++a)
    for (int b = 0; b < ntypes; ++b) {
      const int k = a * ntypes + b;
      const double sig = lj[3 * k], eps = lj[3 * k + 1], rc = lj[3 * k + 2];
      t.s2[k] = sig * sig;
      t.e24[k] = 24.0 * eps;
      t.e4[k] = 4.0 * eps;
      t.rc2[k] = rc * rc;
      const double sr6 = std::pow(t.s2[k] / t.rc2[k], 3);
      t.ushift[k] = 4.0 * eps * (sr6 * sr6 - sr6);
    }
}

struct ForceOut {
  double pe = 0, pe_shift = 0, virial = 0;
  double ncand = 0, nin = 0;
};

// Force laws: kLawLJ (the MD step), kLawCapped (relaxation, extension) and
// kLawSoftCore, the soft-core repulsion of initialAnnealing
// (cudaParticleMD.cu:205-262): potentialSC (kernelinline.hh:136-158) gives
// f0 cos(r / rc_sc * pi / 2), zero for r > rc_sc, which MDpairForce applies
// along (r_i - r_j) / r for pairs inside the LJ cutoff.
enum ForceLaw { kLawLJ = 0, kLawCapped = 1, kLawSoftCore = 2 };

// Pair force of MDpairForce<potentialLJ> (kerneltemplate.hh:530-564,
// kernelinline.hh:86-96) in FP64: F_i = sum_j 24 eps (s/r)^6 (2 (s/r)^6 - 1)/r^2
// * (r_i - r_j), minimum image, truncated at rc, unshifted.  Enumerates the
// 27-cell stencil of each atom's cell exactly as calcF_IJpairWithBlock_F4
// (kerneltemplate.hh:229-294) does, full shell, i != j.
// Energies are sum_{i<j} (counted as half of each ordered pair).
void compute_forces(const double *r3, const uint32_t *type, uint32_t N, const double *L,
                    const Grid &g, const uint32_t *nbr, const uint32_t *start,
                    const uint32_t *members, const uint32_t *cid, const LJTable &t,
                    double *F3, double *pe_atom, ForceOut &out, int law = kLawLJ,
                    double sc_rc = 0, double sc_f0 = 0) {
  const bool capped = law == kLawCapped;
  double pe = 0, pes = 0, vir = 0, nc = 0, ni = 0;
  const int nt = t.ntypes;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : pe, pes, vir, nc, ni)
  for (long ii = 0; ii < (long)N; ++ii) {
    const uint32_t i = (uint32_t)ii;
    const uint32_t I = cid[i];
    const double xi = r3[3 * i], yi = r3[3 * i + 1], zi = r3[3 * i + 2];
    const int ti = (int)type[i];
    double fx = 0, fy = 0, fz = 0, ui = 0;
    for (int L27 = 0; L27 < 27; ++L27) {
      const uint32_t J = nbr[(size_t)I * 27 + L27];
      if (J == 0xffffffffu) continue;
      for (uint32_t s = start[J]; s < start[J + 1]; ++s) {
        const uint32_t j = members[s];
        if (j == i) continue;
        nc += 1;
        double dx = xi - r3[3 * j], dy = yi - r3[3 * j + 1], dz = zi - r3[3 * j + 2];
        if (dx > 0.5 * L[0]) dx -= L[0]; else if (dx < -0.5 * L[0]) dx += L[0];
        if (dy > 0.5 * L[1]) dy -= L[1]; else if (dy < -0.5 * L[1]) dy += L[1];
        if (dz > 0.5 * L[2]) dz -= L[2]; else if (dz < -0.5 * L[2]) dz += L[2];
        const double r2 = dx * dx + dy * dy + dz * dz;
        const int k = ti * nt + (int)type[j];
        if (law == kLawSoftCore) {
          const double r = std::sqrt(r2);
          if (r2 < t.rc2[k] && r <= sc_rc) {
            const double f = sc_f0 * std::cos(r / sc_rc * M_PI / 2) / r;
            fx += f * dx;
            fy += f * dy;
            fz += f * dz;
          }
          continue;
        }
        if (r2 < t.rc2[k]) {
          ni += 1;
          // relaxation force (extension): r^2 floored at (sigma/2)^2 so that
          // overlapping random starts give finite forces
          const double r2f = capped ? std::max(r2, 0.25 * t.s2[k]) : r2;
          const double sr2 = t.s2[k] / r2f;
          const double sr6 = sr2 * sr2 * sr2;
          const double f = t.e24[k] * sr6 * (2.0 * sr6 - 1.0) / r2f;
          fx += f * dx;
          fy += f * dy;
          fz += f * dz;
          const double u = t.e4[k] * (sr6 * sr6 - sr6);
          ui += 0.5 * u;
          pes += 0.5 * (u - t.ushift[k]);
          vir += 0.5 * f * r2;
        }
      }
    }
    F3[3 * i] = fx;
    F3[3 * i + 1] = fy;
    F3[3 * i + 2] = fz;
    if (pe_atom) pe_atom[i] = ui;
    pe += ui;
  }
  out.pe = pe;
  out.pe_shift = pes;
  out.virial = vir;
  out.ncand = nc;
  out.nin = ni;
}

// applyPeriodicCondition_F4 (kernelfuncs.cu:87-139) in FP64: shift by an
// integer number of box lengths into [c0, c1).
inline double wrap1(double x, double c0, double c1) {
  const double L = c1 - c0;
  const double d0 = c0 - x;
  if (d0 > 0) x += (double)((int)(d0 / L) + 1) * L;
  const double d1 = x - c1;
  if (d1 >= 0) x -= (double)((int)(d1 / L) + 1) * L;
  return x;
}

struct System {
  uint32_t N = 0;
  float cell6[6];
  double lo[3], hi[3], L[3];
  float rc_grid = 2.5f;
  Grid g;
  LJTable t;
  std::vector<double> r, v, F, Fold, mass, pe_atom;
  std::vector<uint32_t> type, cid, start, members, nbr;
  double xi = 0;       // Gaussian thermostat friction, carried between steps
  double nr_tol = 1e-8; // Newton-Raphson tolerance (GaussianThermo::_e)
  int nr_iters = 0;
  ForceOut fo;
};

void build_cells(System &s) {
  std::vector<uint32_t> &cid = s.cid;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < (long)s.N; ++i) {
    // The reference bins the FP32 copy of the position (float4 r).
    cid[i] = cell_of(s.g, (float)s.r[3 * i], (float)s.r[3 * i + 1], (float)s.r[3 * i + 2]);
  }
  cell_list(cid.data(), nullptr, s.N, s.g.ncells, s.start.data(), s.members.data());
}

void forces(System &s, int law = kLawLJ, double sc_rc = 0, double sc_f0 = 0) {
  build_cells(s);
  compute_forces(s.r.data(), s.type.data(), s.N, s.L, s.g, s.nbr.data(), s.start.data(),
                 s.members.data(), s.cid.data(), s.t, s.F.data(), s.pe_atom.data(), s.fo, law,
                 sc_rc, sc_f0);
}

void wrap_all(System &s) {
#pragma omp parallel for schedule(static)
  for (long i = 0; i < (long)s.N; ++i)
    for (int k = 0; k < 3; ++k) s.r[3 * i + k] = wrap1(s.r[3 * i + k], s.lo[k], s.hi[k]);
}

// propagateVelocityVerlet_F4 (kernelfuncs.cu:333-367):
//   v += (F + Fold) dt / 2m ;  r += v dt + F dt^2 / 2m ;  Fold = F
void step_vv(System &s, double dt) {
#pragma omp parallel for schedule(static)
  for (long i = 0; i < (long)s.N; ++i) {
    const double h = 0.5 * dt / s.mass[i];
    for (int k = 0; k < 3; ++k) {
      const size_t q = 3 * i + k;
      s.v[q] += (s.F[q] + s.Fold[q]) * h;
      s.r[q] += s.v[q] * dt + s.F[q] * h * dt;
      s.Fold[q] = s.F[q];
    }
  }
}

double sum_mv2(const System &s) {
  double acc = 0;
#pragma omp parallel for schedule(static) reduction(+ : acc)
  for (long i = 0; i < (long)s.N; ++i)
    acc += s.mass[i] * (s.v[3 * i] * s.v[3 * i] + s.v[3 * i + 1] * s.v[3 * i + 1] +
                        s.v[3 * i + 2] * s.v[3 * i + 2]);
  return acc;
}

double sum_fv(const System &s) {
  double acc = 0;
#pragma omp parallel for schedule(static) reduction(+ : acc)
  for (long i = 0; i < (long)(3 * s.N); ++i) acc += s.F[i] * s.v[i];
  return acc;
}

// GaussianThermo::TimeEvolution (GaussianThermo.cu:29-77) with its kernels
// calcGaussianThermoA1_F4, calcGaussianThermoFoverF_F4 and
// propagateVelocityVerletGaussianThermo_F4 (kernelfuncs.cu:372-471), in FP64:
//   A  = v + (F+Fold) dt/2m - v xi dt/2 ;  v <- v + (F+Fold) dt/2m
//   repeat: f = A - (1 + xi dt/2) v ; f' = -dt/2 (xi + (F - 2 xi m v) v / sum mv^2) - 1
//           v -= f/f' ; xi = sum F.v / sum m v^2          until rms(f/f') <= tol
//   r += v (dt - xi dt^2/2) + F dt^2/2m ; Fold = F
// sum F.v is the full sum (innerProduct_F4's overwrite is not reproduced).
// Returns the iteration count, or -1 where the reference gives up (> 51).
int step_gauss(System &s, double dt) {
  std::vector<double> A(3 * (size_t)s.N);
  const double xi_old = s.xi;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < (long)s.N; ++i) {
    const double h = 0.5 * dt / s.mass[i];
    for (int k = 0; k < 3; ++k) {
      const size_t q = 3 * i + k;
      const double vn = s.v[q] + (s.F[q] + s.Fold[q]) * h;
      A[q] = vn - s.v[q] * xi_old * dt * 0.5;
      s.v[q] = vn;
    }
  }
  double mv2inv = 1.0 / sum_mv2(s);
  int it = 0;
  double rms = 0;
  do {
    if (it++ > 50) return -1;
    double acc = 0;
    const double xi = s.xi;
#pragma omp parallel for schedule(static) reduction(+ : acc)
    for (long i = 0; i < (long)s.N; ++i) {
      for (int k = 0; k < 3; ++k) {
        const size_t q = 3 * i + k;
        const double vq = s.v[q];
        const double f1 = A[q] - (0.5 * dt * xi + 1.0) * vq;
        const double f2 = -0.5 * dt * (xi + (s.F[q] - 2.0 * xi * s.mass[i] * vq) * vq * mv2inv) - 1.0;
        const double d = f1 / f2;
        s.v[q] = vq - d;
        acc += d * d;
      }
    }
    rms = std::sqrt(acc / (3.0 * s.N));
    mv2inv = 1.0 / sum_mv2(s);
    s.xi = sum_fv(s) * mv2inv;
  } while (rms > s.nr_tol);
  const double xi = s.xi;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < (long)s.N; ++i) {
    const double h2 = 0.5 * dt * dt / s.mass[i];
    for (int k = 0; k < 3; ++k) {
      const size_t q = 3 * i + k;
      s.r[q] += s.v[q] * (dt - xi * 0.5 * dt * dt) + s.F[q] * h2;
      s.Fold[q] = s.F[q];
    }
  }
  s.nr_iters = it;
  return it;
}

}  // namespace

extern "C" {

// ---- stateless helpers -------------------------------------------------------

int orc_grid_p(const float *cell6, float rc, int periodic, uint32_t *n3, float *len3);
int orc_bin_p(const float *r4, uint32_t N, const float *cell6, float rc, int periodic,
              uint32_t *cid);

int orc_grid(const float *cell6, float rc, uint32_t *n3, float *len3) {
  return orc_grid_p(cell6, rc, 1, n3, len3);
}

int orc_grid_p(const float *cell6, float rc, int periodic, uint32_t *n3, float *len3) {
  Grid g;
  if (make_grid(cell6, rc, g, periodic)) return -1;
  for (int k = 0; k < 3; ++k) {
    n3[k] = g.n[k];
    len3[k] = g.len[k];
  }
  return 0;
}

int orc_neighbor_table(const float *cell6, float rc, int periodic, uint32_t *out) {
  Grid g;
  if (make_grid(cell6, rc, g, periodic)) return -1;
  neighbor_table(g, periodic, out);
  return 0;
}

int orc_bin(const float *r4, uint32_t N, const float *cell6, float rc, uint32_t *cid) {
  return orc_bin_p(r4, N, cell6, rc, 1, cid);
}

int orc_bin_p(const float *r4, uint32_t N, const float *cell6, float rc, int periodic,
              uint32_t *cid) {
  Grid g;
  if (make_grid(cell6, rc, g, periodic)) return -1;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < (long)N; ++i) cid[i] = cell_of(g, r4[4 * i], r4[4 * i + 1], r4[4 * i + 2]);
  return 0;
}

int orc_cell_list(const uint32_t *cid, const float *z, uint32_t N, uint32_t ncells,
                  uint32_t *start, uint32_t *members) {
  cell_list(cid, z, N, ncells, start, members);
  return 0;
}

// Wrap FP32 positions exactly as applyPeriodicCondition_F4 does in FP32
// (used to check the device wrap bit for bit).
void orc_wrap_f32(float *r4, uint32_t N, const float *cell6) {
  const float c0[3] = {cell6[0], cell6[2], cell6[4]};
  const float c1[3] = {cell6[1], cell6[3], cell6[5]};
  for (uint32_t i = 0; i < N; ++i)
    for (int k = 0; k < 3; ++k) {
      const float L = c1[k] - c0[k];
      float x = r4[4 * i + k];
      const float d0 = c0[k] - x;
      if (d0 > 0) {
        const int l0 = static_cast<int>(d0 / L) + 1;
        x += l0 * L;
      }
      const float d1 = x - c1[k];
      if (d1 >= 0) {
        const int l1 = static_cast<int>(d1 / L) + 1;
        x -= l1 * L;
      }
      r4[4 * i + k] = x;
    }
}

// ---- stateful system ---------------------------------------------------------

// lj: ntypes*ntypes triples (sigma, epsilon, rc) in row-major type order.
// rc_grid is the cell-grid cutoff passed to setupCutoffBlock (the largest rc).
void *orc_create(uint32_t N, const float *cell6, float rc_grid, const double *lj, int ntypes) {
  if (ntypes < 1 || ntypes > kMaxTypes) return nullptr;
  System *s = new System;
  s->N = N;
  std::memcpy(s->cell6, cell6, sizeof(float) * 6);
  for (int k = 0; k < 3; ++k) {
    s->lo[k] = cell6[2 * k];
    s->hi[k] = cell6[2 * k + 1];
    s->L[k] = s->hi[k] - s->lo[k];
  }
  s->rc_grid = rc_grid;
  if (make_grid(cell6, rc_grid, s->g)) {
    delete s;
    return nullptr;
  }
  make_table(lj, ntypes, s->t);
  s->r.assign(3 * (size_t)N, 0);
  s->v.assign(3 * (size_t)N, 0);
  s->F.assign(3 * (size_t)N, 0);
  s->Fold.assign(3 * (size_t)N, 0);
  s->mass.assign(N, 1.0);
  s->pe_atom.assign(N, 0);
  s->type.assign(N, 0);
  s->cid.assign(N, 0);
  s->start.assign(s->g.ncells + 1, 0);
  s->members.assign(N, 0);
  s->nbr.assign((size_t)s->g.ncells * 27, 0);
  neighbor_table(s->g, 1, s->nbr.data());
  return s;
}

void orc_destroy(void *h) { delete (System *)h; }

void orc_set_state(void *h, const double *r3, const double *v3, const double *mass,
                   const uint32_t *type) {
  System &s = *(System *)h;
  if (r3) std::memcpy(s.r.data(), r3, sizeof(double) * 3 * s.N);
  if (v3) std::memcpy(s.v.data(), v3, sizeof(double) * 3 * s.N);
  if (mass) std::memcpy(s.mass.data(), mass, sizeof(double) * s.N);
  if (type) std::memcpy(s.type.data(), type, sizeof(uint32_t) * s.N);
}

void orc_set_fold(void *h, const double *fold3) {
  System &s = *(System *)h;
  std::memcpy(s.Fold.data(), fold3, sizeof(double) * 3 * s.N);
}
void orc_set_xi(void *h, double xi) { ((System *)h)->xi = xi; }
void orc_set_tol(void *h, double tol) { ((System *)h)->nr_tol = tol; }

// Forces at the current positions.  out[0..4] = PE (unshifted), PE (shifted
// by U(rc) per pair, the quantity truncated-force dynamics conserve together
// with KE), virial sum_{i<j} r.f, ordered candidate pairs over the 27-cell
// stencil, ordered pairs inside the cutoff.
void orc_forces(void *h, double *out5) {
  System &s = *(System *)h;
  forces(s);
  if (out5) {
    out5[0] = s.fo.pe;
    out5[1] = s.fo.pe_shift;
    out5[2] = s.fo.virial;
    out5[3] = s.fo.ncand;
    out5[4] = s.fo.nin;
  }
}

// Reference step order (testMD2.cu:149-168 without the temperature policy):
// cell build + force, time evolution, periodic wrap.  The first call must be
// preceded by clearing Fold (cudaParticleVV::clearForce); orc_create does.
// mode 0: velocity Verlet (NVE), 1: Gaussian isokinetic.
// energy_out (optional, steps x 3): KE, PE, PE_shift of time t_k of each
// step: PE from the force evaluation at r(t_k) and KE from v(t_k), the
// velocity TimeEvolution produces in the same step (cudaParticleVV.hh:27-39:
// v(t) = v(t - dt) + dt (F(t) + F(t - dt)) / 2m).  Returns 0, or -1 if the
// Newton-Raphson loop did not converge.
int orc_run(void *h, uint32_t steps, double dt, int mode, double *energy_out) {
  System &s = *(System *)h;
  for (uint32_t k = 0; k < steps; ++k) {
    forces(s);
    if (mode == 0) {
      step_vv(s, dt);
    } else {
      if (step_gauss(s, dt) < 0) return -1;
    }
    if (energy_out) {
      energy_out[3 * k] = 0.5 * sum_mv2(s);
      energy_out[3 * k + 1] = s.fo.pe;
      energy_out[3 * k + 2] = s.fo.pe_shift;
    }
    wrap_all(s);
  }
  return 0;
}

// Extension (not in the reference): steepest-descent relaxation used to
// prepare random Kob-Andersen configurations.  Each iteration evaluates the
// relaxation force (pair distance floored at sigma/2) and moves every atom by
// F * min(alpha, max_disp / |F|): a plain gradient step, capped at max_disp
// per atom so that overlapping pairs separate without flinging atoms away.
void orc_steepest_descent(void *h, uint32_t iters, double alpha, double max_disp) {
  System &s = *(System *)h;
  for (uint32_t it = 0; it < iters; ++it) {
    forces(s, kLawCapped);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)s.N; ++i) {
      const double fx = s.F[3 * i], fy = s.F[3 * i + 1], fz = s.F[3 * i + 2];
      const double f = std::sqrt(fx * fx + fy * fy + fz * fz);
      const double g = f * alpha > max_disp ? max_disp / f : alpha;
      s.r[3 * i] += g * fx;
      s.r[3 * i + 1] += g * fy;
      s.r[3 * i + 2] += g * fz;
    }
    wrap_all(s);
  }
}

// adjustVelocity_F4 / adjustVelocity_VD (kernelfuncs.cu:546-699), called by
// adjustVelocities (cudaParticleMD.cu:177-198, GaussianThermo.cu:98-119):
// per axis, FP64 mean and variance over all atoms, then
// v = (v - mean) * v1 / sqrt(variance).
void orc_adjust_velocities(void *h, double v1) {
  System &s = *(System *)h;
  double m[3] = {0, 0, 0}, q[3] = {0, 0, 0};
  for (uint32_t i = 0; i < s.N; ++i)
    for (int k = 0; k < 3; ++k) {
      m[k] += s.v[3 * i + k];
      q[k] += s.v[3 * i + k] * s.v[3 * i + k];
    }
  double f[3];
  for (int k = 0; k < 3; ++k) {
    m[k] /= s.N;
    f[k] = v1 / std::sqrt(q[k] / s.N - m[k] * m[k]);
  }
  for (uint32_t i = 0; i < s.N; ++i)
    for (int k = 0; k < 3; ++k) s.v[3 * i + k] = (s.v[3 * i + k] - m[k]) * f[k];
}

// scaleTemp (cudaParticleMD.cu:168-175, GaussianThermo.cu:89-96): T0 = sum m
// v^2 / (3 N kB), v *= sqrt((3N - 1) / (3N) T / T0).  Returns the factor.
double orc_scale_temp(void *h, double T, double kB) {
  System &s = *(System *)h;
  const double T0 = sum_mv2(s) / (3.0 * s.N * kB);
  const double f = std::sqrt((3.0 * s.N - 1) / (3.0 * s.N) * T / T0);
  for (double &x : s.v) x *= f;
  return f;
}

// Soft-core force of initialAnnealing (see kLawSoftCore) at the current
// positions.
void orc_forces_softcore(void *h, double rc, double f0) {
  System &s = *(System *)h;
  forces(s, kLawSoftCore, rc, f0);
}

// constTemp (cudaParticleMD.cu:140-155) with correctConstTemp_F4
// (kernelfuncs.cu:533-544): lambda = sum F.v / sum m v^2, F -= lambda m v.
// Returns lambda.
double orc_const_temp(void *h) {
  System &s = *(System *)h;
  const double lam = sum_fv(s) / sum_mv2(s);
  if (lam != 0)
    for (uint32_t i = 0; i < s.N; ++i)
      for (int k = 0; k < 3; ++k) s.F[3 * i + k] -= lam * s.mass[i] * s.v[3 * i + k];
  return lam;
}

// The Euler step of initialAnnealing (cudaParticleMD.cu:271-277): calcA_F4
// (kernelfuncs.cu:70-82), propagateEuler_F4 (kernelfuncs.cu:174-192: r += v dt
// with the old v, then v += a dt) and the periodic wrap.
void orc_euler(void *h, double dt) {
  System &s = *(System *)h;
  for (uint32_t i = 0; i < s.N; ++i)
    for (int k = 0; k < 3; ++k) {
      const size_t q = 3 * i + k;
      s.r[q] += s.v[q] * dt;
      s.v[q] += s.F[q] / s.mass[i] * dt;
    }
  wrap_all(s);
}

// cudaParticleMD::initialAnnealing (cudaParticleMD.cu:205-325): anealstep
// soft-core Euler steps with the range growing to rc (rc (i + 1) / anealstep),
// each with constTemp; a rescale to T; Fold cleared; anealstep LJ
// velocity-Verlet steps with constTemp; a final rescale.
void orc_initial_annealing(void *h, uint32_t anealstep, double dt, double rc, double f0,
                           double T, double kB) {
  System &s = *(System *)h;
  for (uint32_t i = 0; i < anealstep; ++i) {
    forces(s, kLawSoftCore, rc * (i + 1) / anealstep, f0);
    orc_const_temp(h);
    orc_euler(h, dt);
  }
  orc_scale_temp(h, T, kB);
  std::fill(s.Fold.begin(), s.Fold.end(), 0.0);
  for (uint32_t i = 0; i < anealstep; ++i) {
    forces(s);
    orc_const_temp(h);
    step_vv(s, dt);
    wrap_all(s);
  }
  orc_scale_temp(h, T, kB);
}

double orc_kinetic(void *h) { return 0.5 * sum_mv2(*(System *)h); }
double orc_get_xi(void *h) { return ((System *)h)->xi; }
int orc_get_nr_iters(void *h) { return ((System *)h)->nr_iters; }

void orc_get(void *h, int field, double *out) {
  System &s = *(System *)h;
  const size_t n3 = 3 * (size_t)s.N;
  switch (field) {
    case 0: std::memcpy(out, s.r.data(), sizeof(double) * n3); break;
    case 1: std::memcpy(out, s.v.data(), sizeof(double) * n3); break;
    case 2: std::memcpy(out, s.F.data(), sizeof(double) * n3); break;
    case 3: std::memcpy(out, s.Fold.data(), sizeof(double) * n3); break;
    case 4: std::memcpy(out, s.pe_atom.data(), sizeof(double) * s.N); break;
    default: break;
  }
}

int orc_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
