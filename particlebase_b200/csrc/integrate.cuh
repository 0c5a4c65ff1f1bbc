// Time integration and reductions, for one system or many packed systems.
//
// Every CUDA block works on a contiguous atom range of ONE system (the block
// map below), and every per-system sum is finished by that system's last
// block, adding the block partials in block order.  The arithmetic an atom
// sees therefore depends only on its own system, never on which other
// systems share the launch: a system gives bit-identical results alone and
// in a batch.
#pragma once

#include "common.cuh"

namespace pb {

constexpr int kIntThreads = 256;  // threads per integration block
constexpr int kIntAtoms = 1024;   // atoms per integration block (4 per thread, strided)

// Device-resident scalars of one system.  Reductions are finished on the
// device (last-block pattern), so a step never needs a host round trip.
struct DevScalars {
  double xi_old;      // Gaussian friction used by the current step's A term
  double xi_new;      // friction solved this step
  double sum_fa;      // sum F . A
  double sum_ma2;     // sum m A^2
  double mv2;         // sum m v^2 after the last update
  double pe, pe_shift, virial;   // from the last force call with energy
  double vstat[6];    // sum v, sum v^2 per axis (adjustVelocities)
  double fv;          // sum F . v (constTemp)
  double npairs;      // ordered pairs inside the cutoff (last force with energy)
  unsigned int counter[4];
};

// Integration view of one system.
struct SysInt {
  uint32_t atom0, natoms;  // atom range in the packed arrays
  uint32_t vd0;            // start of this system's FP64 velocity planes (x, y, z)
  uint32_t blk0, nblk;     // its integration blocks
  float dt;
  float c0[3], c1[3], L[3];  // box for the wrap
};

// Block b of an integration launch covers atoms [i0, i0 + n) of system sys,
// n <= kIntAtoms; it is block `k` of that system (i0 = first atom + k kIntAtoms).
struct BlockMap {
  uint32_t sys, i0, n, k;
};

struct IntegrateArgs {
  float4 *r;
  float4 *v;          // FP32 velocities (nullptr when vd is used)
  double *vd;         // FP64 velocities, per-system SoA planes
  const float4 *F;    // F(t)
  const float4 *Fold; // F(t - dt)
  const float *minv;
  const float *mass;
  const SysInt *sys;
  const BlockMap *map;
  uint32_t nblocks;
  int wrap;
  DevScalars *sc;     // per system
  double *partials;   // >= 8 doubles per block
  uint32_t *status;   // status bits, one word per system
  uint32_t *steps_left;  // per system: steps still to run, 0 = finished and left
                         // unchanged; decremented by each VV / Gaussian step
                         // (nullptr: no limit)
};

cudaError_t launch_vv(const IntegrateArgs &a, cudaStream_t s);
cudaError_t launch_gauss(const IntegrateArgs &a, cudaStream_t s);
cudaError_t launch_wrap(const IntegrateArgs &a, cudaStream_t s);
cudaError_t launch_mv2(const IntegrateArgs &a, cudaStream_t s);
cudaError_t launch_fv(const IntegrateArgs &a, cudaStream_t s);
// Per-system factors / v1 values (device arrays, one double per system).
cudaError_t launch_scale(const IntegrateArgs &a, const double *factors, cudaStream_t s);
cudaError_t launch_adjust(const IntegrateArgs &a, const double *v1, cudaStream_t s);
// Euler step of initialAnnealing (calcA_F4 + propagateEuler_F4,
// kernelfuncs.cu:70-82, 174-192): r += v dt, v += F/m dt, then wrap.
cudaError_t launch_euler(const IntegrateArgs &a, const float4 *F, float dt, cudaStream_t s);
// Steepest-descent move: r += F min(alpha, max_disp / |F|), then wrap.
cudaError_t launch_sd_move(const IntegrateArgs &a, const float4 *F, float alpha, float max_disp,
                           cudaStream_t s);
// F -= lambda[sys] m v on the force buffer `F` (constTemp).
cudaError_t launch_correct_force(const IntegrateArgs &a, float4 *F, const double *lambda,
                                 cudaStream_t s);
// Per-system energy totals from force partials: system s owns partials
// [item0[s], item0[s + 1]) (4 doubles each).
cudaError_t launch_energy_total(const double *partials, const uint32_t *item0, uint32_t nsys,
                                DevScalars *sc, cudaStream_t s);

// Owning system of every atom, written from the block map.
cudaError_t launch_fill_sysid(const BlockMap *map, uint32_t nblocks, uint32_t *sysid,
                              cudaStream_t s);

// State of one system of a new batch that continues a system of an old one.
struct GatherSrc {
  int32_t src;       // old system, or -1 for a new system (zeroed)
  uint32_t o_atom0;  // its first atom in the old arrays
  uint8_t fb0, fb1;  // old force buffer that feeds new F[0] and new F[1]
};

struct GatherArgs {
  const BlockMap *map;  // blocks of the new batch
  const SysInt *sys;    // systems of the new batch
  uint32_t nblocks;
  const GatherSrc *gs;  // per new system
  const float4 *o_r, *o_v, *o_F0, *o_F1;
  const double *o_vd;
  const float *o_minv, *o_mass;
  const uint16_t *o_type;
  float4 *r, *v, *F0, *F1;
  double *vd;
  float *minv, *mass;
  uint16_t *type;
};
// Copy every continuing system's per-atom state, and zero every new system's, in one launch.
cudaError_t launch_gather_state(const GatherArgs &g, cudaStream_t s);

// Host helpers: integration blocks of kIntAtoms atoms aligned to each
// system's first atom.
uint32_t blocks_for(uint32_t natoms);
void make_block_map(const uint32_t *natoms, uint32_t nsys, BlockMap *map, uint32_t *blk0,
                    uint32_t *nblk);

}  // namespace pb
