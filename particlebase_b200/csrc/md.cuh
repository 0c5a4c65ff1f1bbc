// Device data layout of one or many LJ systems packed into shared arrays, and
// the kernel entry points that operate on them.
//
// Layout in HBM (all arrays in particle order unless noted):
//   r      float4[N]   position x, y, z (w unused)           -- cudaParticleBase::r
//   v      float4[N]   velocity (FP32 path), w = 0           -- cudaParticleBase::v
//   vd     double[3N]  velocity, FP64, per-system SoA planes -- GaussianThermo::vd
//   F[2]   float4[N]   force ping-pong: F[cur] is F(t), F[1-cur] is Fold
//   minv   float[N]    1 / mass                               -- cudaParticleBase::minv
//   type   uint16[N]   type id                                -- cudaParticleBase::typeID
//   sysid  uint32[N]   owning system (batched mode only)
// Cell list (rebuilt every step):
//   key    uint32[N]   packed cell key of each atom: cell0 + rank(x,y) * nz + z
//   start  uint32[C+1] first sorted slot of each packed cell (C = all cells)
//   pid    uint32[N]   particle id at each sorted slot (cudaCutoffBlock::pid)
//   slot   uint32[N]   sorted slot of each particle (inverse of pid)
//   rs     float4[N]   sorted positions, w = type id bits (cudaSortedPositions::r_s)
//   xs, ys, zs float, ts uint32 [M]  SoA mirrors of rs; system s at mirror0(s) + k,
//          mirror0 a multiple of 4 (M = sum of the systems' sizes rounded up to 4, + 4)
// Cell keys order the (x, y) columns of a box along a Morton (Z-order) curve and
// keep z fastest, so the three z-adjacent cells of a column are contiguous.
#pragma once

#include "common.cuh"

namespace pb {

struct BlockMap;  // integrate.cuh

// One periodic system inside the packed arrays.
struct SysDesc {
  Grid g;
  uint32_t atom0, natoms;   // particle range [atom0, atom0 + natoms)
  uint32_t cell0;           // first packed cell key
  uint32_t col0;            // offset of this system's column tables
  uint32_t vd0;             // offset of this system's FP64 velocity planes (3 * atom0)
  uint32_t lj;              // index of this system's LJ table
  float dt;                 // time step
  uint32_t cap;             // staged-atom capacity of this system's force CTAs
  uint32_t mirror0;         // first slot of this system in the SoA mirrors (multiple of 4)
  uint32_t cap_half;        // staged-atom capacity of the half-shell force CTAs
};

// Work item of the force kernel: one (x, y) column of one system, z cells
// [z0, z1).  Items are listed in column-Morton order.  The packed key of z cell
// 0 of the 3 x 3 neighbour columns (x offset outer, y offset inner, each
// -1, 0, +1, periodic) is precomputed on the host, so a CTA's first global
// loads are the cell starts it stages.
struct ForceItem {
  uint32_t sys;
  uint32_t col;         // column rank within the system
  uint16_t z0, z1;
  uint16_t cx, cy;      // column coordinates (frame shifts on the top faces)
  uint32_t kbase[9];
};

struct CellBufs {
  const float4 *r;
  const uint16_t *type;
  const uint32_t *sysid;     // nullptr: every atom belongs to system 0
  const SysDesc *sys;
  const uint32_t *colrank;   // per system: reference column (d0 * ny + d1) -> rank
  uint32_t N;
  uint32_t ncells;           // packed cells over all systems
  uint32_t *key, *within, *count, *start, *tilesum;
  uint32_t *pid_tmp, *pid, *slot;
  // two-kernel build (bucket == nullptr: the six-kernel counting sort)
  uint32_t *bucket;          // per cell, bucket_cap member ids in ticket order
  uint32_t bucket_cap;       // at least 32
  uint2 *ovf;                // (cell, atom) of the members past bucket_cap; N entries
  uint32_t *tcount;          // atoms per 64-cell tile
  uint32_t ntile;
  uint32_t tile_atoms;       // members a k_canon_tiles block stages in shared memory
  uint32_t *ctl;             // [0] overflow entries, [1] finished k_canon_tiles blocks
  float4 *rs;
  // structure-of-arrays mirrors of rs (nullptr: not written); system s's
  // sorted atom k sits at mirror0 + k, so 16-byte runs align the same way
  // whether the system runs alone or in a batch
  float *xs, *ys, *zs;
  uint32_t *ts;
  uint32_t *status;
};

struct ForceBufs {
  const float4 *rs;
  const float *xs, *ys, *zs;  // SoA mirrors of rs (per-system aligned, see CellBufs)
  const uint32_t *ts;
  const uint32_t *start;     // packed cell starts
  const uint32_t *pid;
  const SysDesc *sys;
  const uint32_t *colxy;     // per system: rank -> reference column (d0 * ny + d1)
  const uint32_t *colrank;   // per system: reference column -> rank
  const LJTable *lj;
  const ForceItem *items;
  uint32_t nitems;
  int cap;                   // shared-memory capacity of the launch (max over systems)
  float4 *F;                 // force output, particle order
  double *partials;          // per-item energy partials (4 doubles per item)
  uint32_t *status;
  const uint32_t *steps_left;  // per system; 0 = finished, skipped (nullptr: all run)
  float sc_rc, sc_f0;          // soft-core force law: range and strength
  uint32_t *queue;           // [0] next unclaimed item, [1] CTAs done claiming; zero
                             // between launches (the last CTA resets them)
  // half-shell kernel (force_half.cu)
  unsigned long long *facc;  // fixed-point force sums (2^-32 units), planes x, y, z of
                             // nacc entries indexed by sorted slot; zero between calls
  unsigned long long *fbig;  // the same in units of 1/2, for shares of 2^22 and more
  uint32_t nacc;             // atoms of all systems
  int cap_half;              // stage capacity of the launch (max over systems)
  const BlockMap *map;       // integration blocks (per-system atom ranges)
  uint32_t nblocks;
  uint32_t wait_polls;       // bound of the hand-off waits, 0 = default
  uint32_t test_flags;       // bit 0: withhold the first hand-off (failure-detection test)
};

// Verlet neighbour list of one system: row s holds the build-time sorted
// slots of the atoms within the list radius of the atom that sat in slot s
// when the list was built, column-major (entry k of row s at idx[k * N + s]).
struct NlistBufs {
  const float4 *r;           // positions, particle order
  const float4 *rs;          // sorted positions (build)
  const uint32_t *pid, *start, *key, *colxy, *colrank;  // cell list (build)
  const uint16_t *type;
  const SysDesc *sys;        // the one system
  const LJTable *lj;
  uint32_t N, cap;           // atoms; entries per row
  float rl2;                 // list radius squared (build)
  float skin;                // list radius minus the force cutoff
  uint32_t *idx, *cnt, *atom;  // rows, row counts, particle of each row
  float4 *rl;                // current positions in row order (refreshed every force call)
  float4 *r0;                // positions at the build, row order
  uint32_t *maxcnt;          // build: largest row count (reset by the caller)
  float4 *F;                 // force output, particle order
  double *partials;          // per-block energy partials (4 doubles per block)
  uint32_t *status;
};

// Launchers (return cudaError_t of the launch).
cudaError_t launch_cell_build(const CellBufs &b, cudaStream_t s);
cudaError_t launch_force(const ForceBufs &b, int nt_max, bool energy, bool acc64,
                         int block_threads, cudaStream_t s);
// Half-shell force (each pair once, fixed-point sums) followed by the
// conversion of the sums to F; FP32 pair arithmetic.
cudaError_t launch_force_half(const ForceBufs &b, int nt_max, bool energy, cudaStream_t s);
// Relaxation force for steepest descent: pair distance floored at sigma/2.
cudaError_t launch_force_capped(const ForceBufs &b, int nt_max, cudaStream_t s);
// Soft-core force f0 cos(pi r / 2 sc_rc) along r (potentialSC), for annealing.
cudaError_t launch_force_softcore(const ForceBufs &b, int nt_max, cudaStream_t s);
// Neighbour list: build from the cell list; forces over the list.
cudaError_t launch_nlist_build(const NlistBufs &b, cudaStream_t s);
// (launch_nlist_force refreshes rl from r before the pair loop)
cudaError_t launch_nlist_force(const NlistBufs &b, int nt_max, bool energy, bool acc64,
                               cudaStream_t s);
uint32_t nlist_blocks(uint32_t N);  // blocks (energy partials) of launch_nlist_force
// Pair counts per distance bin over all unordered pairs (g(r)); counts must
// be zeroed by the caller; rnum <= gr_max_bins().
cudaError_t launch_gr(const float4 *r, uint32_t N, const float L[3], float inv, uint32_t rnum,
                      unsigned long long *counts, cudaStream_t s);
uint32_t gr_max_bins();

}  // namespace pb
