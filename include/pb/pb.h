/*
 * particlebase_b200 — C ABI of the B200-native Lennard-Jones cell-list step.
 *
 * One pb_md handle is one periodic MD system resident on the current CUDA
 * device: the state the reference keeps in a cudaParticleMD / cudaParticleVV /
 * GaussianThermo object (cudaParticleBase.hh:29-226, cudaCutoffBlock.hh:28-133,
 * cudaSortedPositions.hh:6-36, cudaParticleMD.hh:32-194, GaussianThermo.hh:14-90).
 * The C++ classes in particlebase_b200/shim/ (same names and methods as the
 * reference) are a thin layer over these functions, so the reference's
 * testMD drivers compile against them unchanged.
 *
 * Conventions
 *  - Every function returns pb_status (0 = success) and never calls exit();
 *    pb_md_last_error() describes the last failure of a handle.
 *  - Plain pointers and sizes only.  Host arrays are read or written
 *    synchronously with respect to the handle's stream.
 *  - All device work of a handle is issued on its stream (default: a stream
 *    the handle creates); pb_md_set_stream() selects another one.
 *  - Positions, velocities and forces use the reference's layouts: float4
 *    per particle (x, y, z, w) in particle order; FP64 velocities of the
 *    Gaussian thermostat as three planes x[N], y[N], z[N].
 */
#ifndef PB_PB_H
#define PB_PB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum pb_status {
  PB_OK = 0,
  PB_ERR_ARG = 1,          /* invalid argument or size */
  PB_ERR_CUDA = 2,         /* a CUDA call failed */
  PB_ERR_STATE = 3,        /* call out of order (e.g. force before cells) */
  PB_ERR_NOCONVERGE = 4,   /* thermostat solve failed (reference: exit(0)) */
  PB_ERR_UNSUPPORTED = 5,  /* feature outside this build (e.g. open boundaries) */
  PB_ERR_OOM = 6,          /* device allocation or HBM budget exceeded */
  PB_ERR_DEVICE = 7,       /* a kernel reported a status bit (see pb_md_status) */
  PB_ERR_NOTFOUND = 8      /* unknown job / field */
} pb_status;

/* Host particle record, binary-compatible with the reference's ParticleBase
 * (ParticleBase.hh:10-18): double r[3], m, v[3]; bool isFixed; double a[3];
 * uint32_t type. */
typedef struct pb_particle {
  double r[3];
  double m;
  double v[3];
  uint8_t is_fixed;
  double a[3];
  uint32_t type;
} pb_particle;

typedef struct pb_md pb_md;

/* Creation flags */
#define PB_MD_VEL_FP64 0x1u   /* keep velocities in FP64 planes (GaussianThermo::vd) */
#define PB_MD_ACC_FP64 0x2u   /* accumulate per-atom force sums in FP64 */
#define PB_MD_HALF_SHELL 0x4u /* evaluate every unordered pair once (Newton's third law)
                                 with exact fixed-point force sums, instead of every ordered
                                 pair as calcF_IJpairWithBlock_F4 does (the default);
                                 ignored with PB_MD_ACC_FP64 */

/* Fields for pb_md_get / pb_md_set */
typedef enum pb_field {
  PB_FIELD_R = 0,          /* float4[N]   positions                       (get/set) */
  PB_FIELD_V = 1,          /* float4[N]   velocities (FP32 path)          (get/set) */
  PB_FIELD_VD = 2,         /* double[3N]  velocities, FP64 planes         (get/set) */
  PB_FIELD_F = 3,          /* float4[N]   force F(t)                      (get/set) */
  PB_FIELD_FOLD = 4,       /* float4[N]   previous force (VV Fold)        (get/set) */
  PB_FIELD_MINV = 5,       /* float[N]    1/mass                          (get/set) */
  PB_FIELD_TYPE = 6,       /* uint16[N]   type id                         (get/set) */
  PB_FIELD_CELL_OF = 7,    /* uint32[N]   reference cell id of each atom  (get) */
  PB_FIELD_PID = 8,        /* uint32[N]   particle id per sorted slot     (get) */
  PB_FIELD_CELL_START = 9, /* uint32[C+1] first slot of each cell, in key order (get) */
  PB_FIELD_CELL_KEY = 10,  /* uint32[C]   key of each reference cell id   (get) */
  PB_FIELD_NEIGHBORS = 11, /* uint32[27C] 27-neighbour table, reference order (get) */
  PB_FIELD_R_SORTED = 12,  /* float4[N]   sorted positions, w = type bits (get) */
  PB_FIELD_MASS = 13       /* float[N]    mass                            (get) */
} pb_field;

/* Energy / reduction results of pb_md_reduce */
typedef struct pb_md_sums {
  double mv2;       /* sum m v^2 (3 N kB T) */
  double fv;        /* sum F . v */
  double pe;        /* potential energy, truncated and unshifted, sum_{i<j} */
  double pe_shift;  /* potential energy shifted by U(rc) per pair (conserved with KE) */
  double virial;    /* sum_{i<j} r_ij . f_ij */
  double xi;        /* Gaussian thermostat friction of the last step */
} pb_md_sums;

/* ---- lifetime ------------------------------------------------------------ */

/* cudaParticleBase::setup + cudaParticleVV::setup + cudaParticleMD::setup +
 * GaussianThermo::setup (cudaParticleBase.cu:18-66, cudaParticleVV.cu:5-8,
 * cudaParticleMD.cu:13-22, GaussianThermo.cu:9-14). */
int pb_md_create(uint32_t n, uint32_t flags, pb_md **out);
/* The destructors (cudaParticleBase.cu:7-16 and siblings). */
int pb_md_destroy(pb_md *h);
/* Issue all work of the handle on `stream` (a cudaStream_t). */
int pb_md_set_stream(pb_md *h, void *stream);
const char *pb_md_last_error(const pb_md *h);
/* Device status bits raised by kernels since the last call (cleared on read). */
#define PB_STATUS_SMEM_OVERFLOW 0x1u   /* a force work item computed from global memory */
#define PB_STATUS_NONFINITE 0x2u       /* a NaN or Inf reached a reduction */
#define PB_STATUS_WAIT_TIMEOUT 0x4u    /* a bounded wait in a kernel gave up */
#define PB_STATUS_CELL_OVERFLOW 0x8u   /* a cell held more atoms than a kernel supports */
#define PB_STATUS_NOCONVERGE 0x10u     /* thermostat solve failed */
#define PB_STATUS_NLIST_OVERFLOW 0x20u /* a neighbour-list row outgrew its capacity */
#define PB_STATUS_STALE_NLIST 0x40u    /* an atom moved more than half the list skin */
int pb_md_status(pb_md *h, uint32_t *bits);

/* ---- set-up ---------------------------------------------------------------- */

/* cudaFrame::setCell (cudaFrame.cu:85-91): xmin, xmax, ymin, ymax, zmin, zmax. */
int pb_md_set_cell(pb_md *h, const float cell6[6]);
/* cudaParticleMD::setLJparams -> _setLJparams (cudaParticleMD.cu:200-202,
 * kernelinline.hh:120-134): (sigma, epsilon) per ordered type pair,
 * ntypes <= 8.  The cutoff is the global rmax2 (pb_md_set_rmax2). */
int pb_md_set_lj(pb_md *h, const float *sigma_eps, uint32_t ntypes);
/* Extension: (sigma, epsilon, rc) per type pair; per-pair cutoffs. */
int pb_md_set_lj_cut(pb_md *h, const float *sigma_eps_rc, uint32_t ntypes);
/* Public field cudaParticleMD::rmax2 (cudaParticleMD.hh:160). */
int pb_md_set_rmax2(pb_md *h, float rmax2);
/* Public field cudaParticleMD::kB (cudaParticleMD.hh:94). */
int pb_md_set_kB(pb_md *h, float kB);
/* cudaParticleMD::import (cudaParticleMD.cu:327-336 -> cudaParticleBase.cu:68-117,
 * GaussianThermo.cu:16-28) followed by setM (cudaParticleMD.cu:135-138). */
int pb_md_import(pb_md *h, const pb_particle *p, uint32_t n);
/* Same, from structure-of-arrays host buffers (r3, v3: 3 doubles per atom). */
int pb_md_import_arrays(pb_md *h, const double *r3, const double *v3, const double *mass,
                        const uint32_t *type);
/* cudaParticleMD::setupCutoffBlock -> cudaCutoffBlock::setupCutoffBlock +
 * setupSortedPositions (cudaParticleMD.hh:71-74, cudaCutoffBlock.cu:75-231).
 * periodic = 0: open boundaries as the reference's non-periodic branch --
 * cells of edge rmax, one past each top face, no neighbour across a face
 * (UINT_MAX in the neighbour table), no image in the forces, and steps do
 * not wrap positions (pb_md_wrap still does on request).  Open boxes run on
 * the full-shell cell-list force only: with PB_MD_HALF_SHELL or a neighbour
 * list the call returns PB_ERR_UNSUPPORTED. */
int pb_md_setup_cells(pb_md *h, float rmax, int periodic);
/* Grid of the last setup: cells per axis and cell edge (blocknum, blocklen). */
int pb_md_grid(const pb_md *h, uint32_t n3[3], float len3[3], uint32_t *ncells);

/* ---- the step ------------------------------------------------------------- */

/* cudaParticleMD::calcBlockID (cudaParticleMD.hh:64-67 ->
 * cudaCutoffBlock.cu:233-258, cudaSortedPositions.cu:27-30). */
int pb_md_build_cells(pb_md *h);
/* cudaParticleMD::calcForce (cudaParticleMD.cu:24-69).  flags: PB_FORCE_ENERGY
 * also accumulates PE, shifted PE and virial (FP64) for pb_md_reduce. */
#define PB_FORCE_ENERGY 0x1u
int pb_md_force(pb_md *h, uint32_t flags);
/* Failure-detection test hook (no counterpart in the reference): one force
 * call in which the force kernel's producer warps withhold
 * their first hand-off to the consumer warps, with every hand-off wait bounded
 * by `polls` polls of at most 1 us.  The consumers' wait runs out, the CTAs
 * end early, the call returns PB_OK and the status word carries
 * PB_STATUS_WAIT_TIMEOUT; the forces of that call are not meaningful.  The
 * handle stays usable: the next pb_md_force is complete again. */
int pb_md_force_wait_test(pb_md *h, uint32_t polls);
/* cudaParticleVV::clearForce (cudaParticleVV.cu:10-15): F = Fold = 0. */
int pb_md_clear_force(pb_md *h);
/* cudaParticleVV::TimeEvolution (cudaParticleVV.cu:17-34). */
int pb_md_step_vv(pb_md *h, float dt);
/* GaussianThermo::TimeEvolution (GaussianThermo.cu:29-77), solved on the
 * device in closed form; tol is accepted for interface parity. */
int pb_md_step_gauss(pb_md *h, float dt, double tol);
/* cudaParticleBase::treatPeriodicCondition (cudaParticleBase.cu:175-184). */
int pb_md_wrap(pb_md *h);
/* Whole steps in the reference driver order (testMD2.cu:149-168 without the
 * temperature policy): build cells, force, time evolution with the wrap
 * fused.  mode 0: velocity Verlet, 1: Gaussian.  Captured as a CUDA graph
 * after the first call with the same (dt, mode). */
#define PB_MODE_VV 0
#define PB_MODE_GAUSS 1
int pb_md_run(pb_md *h, float dt, int mode, uint32_t steps);
/* cudaParticleMD::useNList and the public field thickness
 * (cudaParticleMD.hh:41, 167-179): force calls use a Verlet neighbour list of
 * the atoms within rc + thickness (calcF_IJpairWithList_F4,
 * kerneltemplate.hh:135-168), which only pb_md_make_nlist rebuilds; whole
 * steps (pb_md_run) then skip the cell-list build, as testMD4n.cu:175-181 does.
 * thickness < 0 turns the list off.  Single-system handles only.  A force call
 * raises PB_STATUS_STALE_NLIST when an atom moved more than thickness / 2
 * since the build. */
int pb_md_use_nlist(pb_md *h, float thickness);
/* cudaParticleMD::makeNList (cudaParticleMD.cu:338-394): rebuild the cell list
 * and the neighbour list.  The cell edge (pb_md_setup_cells) must be at least
 * rc + thickness, as the reference's cell blocks are; PB_ERR_ARG otherwise.
 * Rows that outgrow their capacity are enlarged and the list built again. */
int pb_md_make_nlist(pb_md *h);
/* Mean and largest row length of the last list build, and the row capacity. */
int pb_md_nlist_info(pb_md *h, double out[3]);
/* cudaCalcGR::setup + calcgr (cudaCalcGR.hh:27-40, cudaCalcGR.cu:85-116,
 * calcGR_F4 at kernelinline.hh:433-449): counts of the unordered pairs of the
 * handle's current positions per distance bin, minimum image, bin
 * j = trunc(r / rstep + 1/2) counted when 0 < j < rnum, rnum = trunc(rmax /
 * rstep) by the reference's FP32 rule.  All pairs, as the reference's pair
 * list over every cell-block pair.  Call with counts = NULL to get *rnum, then
 * with counts[*rnum] (overwritten; bin 0 stays 0).  rnum <= 16384.
 * cudaCalcGR::igr2gr's normalisation g_j = counts_j * Q / (4 j^2 + 1/3),
 * Q = 2 V / (N^2 pi rstep^3), is left to the caller (the drop-in class does it). */
int pb_md_gr(pb_md *h, float rstep, float rmax, uint64_t *counts, uint32_t *rnum);
/* pb_md_run bracketed by CUDA events on the handle's stream; *ms = elapsed. */
int pb_md_run_timed(pb_md *h, float dt, int mode, uint32_t steps, float *ms);

/* Per-phase device time of `steps` eager steps, measured with CUDA events on
 * the handle's stream: ms[0] cell build, ms[1] force, ms[2] time evolution
 * (averages per step). */
int pb_md_profile(pb_md *h, float dt, int mode, uint32_t steps, double ms[3]);
/* Pair statistics of the current cell list: out[0] = ordered candidate pairs
 * over the 27-cell stencil (i != j), out[1] = ordered pairs inside the cutoff
 * counted by the last pb_md_force with PB_FORCE_ENERGY. */
int pb_md_pair_stats(pb_md *h, double out[2]);
/* Kernels one cell build launches: 2 for the bucket build, 6 for the counting
 * sort (the engine picks the faster at pb_md_setup_cells; PB_CELL_BUILD fixes
 * it).  No counterpart in the reference. */
int pb_md_cell_build_kernels(pb_md *h, uint32_t *kernels);

/* ---- reductions and velocity control -------------------------------------- */

/* Sums of the current state: calcMV2 (cudaParticleMD.cu:124-133,
 * GaussianThermo.cu:79-87) in FP64, sum F.v (constTemp, cudaParticleMD.cu:140-155),
 * and PE / virial of the last force call with PB_FORCE_ENERGY. */
int pb_md_reduce(pb_md *h, pb_md_sums *out);
/* cudaParticleMD::calcTemp (cudaParticleMD.hh:89-92): sum m v^2 / (3 N kB). */
int pb_md_temperature(pb_md *h, double *T);
/* scaleTemp (cudaParticleMD.cu:168-175, GaussianThermo.cu:89-96): v *= s. */
int pb_md_scale_velocities(pb_md *h, double s);
/* adjustVelocities (cudaParticleMD.cu:177-198, GaussianThermo.cu:98-119):
 * zero mean per axis, standard deviation v1 per axis. */
int pb_md_adjust_velocities(pb_md *h, double v1);
/* constTemp's force correction (cudaParticleMD.cu:140-155, correctConstTemp_F4
 * kernelfuncs.cu:533-544): F -= lambda m v on the latest force. */
int pb_md_correct_force(pb_md *h, double lambda);
/* initialAnnealing's pieces (cudaParticleMD.cu:205-325): the soft-core force
 * f0 cos(pi r / 2 rc) along r for pairs inside min(rc, the LJ cutoff)
 * (potentialSC, kernelinline.hh:136-158) on the current cell list, and the
 * Euler step with the latest force (calcA_F4 + propagateEuler_F4 + wrap;
 * FP32-velocity handles). */
int pb_md_force_softcore(pb_md *h, float rc, float f0);
int pb_md_step_euler(pb_md *h, float dt);
/* Extension (no counterpart in the reference): steepest-descent relaxation of
 * overlapping starts, `iters` times: cell build, relaxation force (pair
 * distance floored at sigma/2 so forces stay finite), then every atom moves by
 * F min(alpha, max_disp / |F|) and wraps.  F afterwards holds the relaxation
 * force; call pb_md_clear_force before dynamics. */
int pb_md_minimize(pb_md *h, uint32_t iters, float alpha, float max_disp);
/* Gaussian friction xi carried into the next step (GaussianThermo::xi),
 * e.g. when restoring a checkpoint. */
int pb_md_set_xi(pb_md *h, double xi);
/* Mean particle mass m0 of the last import (cudaParticleMD.cu:327-336). */
int pb_md_mean_mass(const pb_md *h, double *m0);

/* ---- state access ----------------------------------------------------------- */

/* getPosition / getForce / getTypeID (cudaParticleBase.cu:119-149) and the
 * other arrays listed in pb_field; `bytes` must equal the field size. */
int pb_md_get(pb_md *h, int field, void *host, size_t bytes);
int pb_md_set(pb_md *h, int field, const void *host, size_t bytes);
int pb_md_field_bytes(const pb_md *h, int field, size_t *bytes);
int pb_md_size(const pb_md *h, uint32_t *n);

/* Host-only (no device work): the cell grid setupCutoffBlock would build for
 * this box and cutoff -- blocknum = (uint32)(L / rmax), blocklen = L / blocknum
 * in FP32 (cudaCutoffBlock.cu:97-101).  Returns PB_ERR_ARG if an axis would
 * have fewer than 3 cells. */
int pb_plan_grid(const float cell6[6], float rmax, uint32_t n3[3], float len3[3]);
/* Host-only: Z-order rank of every (x, y) column, rank[d0 * ny + d1]. */
int pb_plan_columns(uint32_t nx, uint32_t ny, uint32_t *rank);

/* Measured FP32 FMA throughput of the current device (TFLOP/s), from a
 * register-resident FFMA loop timed with CUDA events. */
int pb_peak_fp32(double *tflops);

/* Cell-list build that allocates no device memory.  No counterpart in the
 * reference.  For callers that cannot allocate device memory themselves (a
 * host framework that owns all device memory through its own pool, or a
 * latency-critical loop that must not allocate).  Same result as
 * pb_md_build_cells, bit for bit, with every scratch array held in one static
 * device array of fixed size (see pb_cells_build_noalloc_limits): n at most
 * 131,072 atoms and at most 65,536 cells, larger inputs return PB_ERR_ARG.
 * Device pointers: r4 (float4[n] positions), type (uint16[n] or NULL for all
 * zero); outputs start (uint32[C+1], C from pb_plan_grid, cells in the key
 * order of pb_plan_columns, z fastest), pid (uint32[n]), slot (uint32[n]),
 * rs4 (float4[n] sorted positions, w = type bits).  Enqueued on `stream` (a
 * cudaStream_t, NULL = legacy default) without waiting for it: the outputs
 * are ready when the stream reaches this point, and no host memory of the
 * call is read after it returns.  The first call on a device resolves the
 * static array's device address and keeps it for later calls; make that first
 * call before any stream capture, use one context per device (the CUDA
 * runtime's primary context) and do not reset the device between calls.  All
 * calls share the one array: calls that overlap on the GPU race, so serialise
 * them. */
int pb_cells_build_noalloc(const void *r4, const uint16_t *type, uint32_t n, const float cell6[6],
                           float rmax, uint32_t *start, uint32_t *pid, uint32_t *slot, void *rs4,
                           void *stream);
/* Size limits and static scratch size of pb_cells_build_noalloc. */
int pb_cells_build_noalloc_limits(uint32_t *max_atoms, uint32_t *max_cells, size_t *scratch_bytes);

/* ---- batches of independent systems ----------------------------------------
 *
 * No counterpart in the reference, which runs one system per process
 * (testMD2.cu).  A pb_batch holds many independent periodic LJ systems of
 * any sizes packed into shared device arrays; one launch per kernel advances
 * all of them, and whole steps replay from one CUDA graph.  Every system is
 * computed exactly as a pb_md handle computes it alone (same cell list, same
 * force and integration arithmetic, per-system FP64 sums in the same order):
 * its results are bit-identical alone and in any batch.  Systems are
 * numbered 0 .. nsys-1 in creation order. */
typedef struct pb_batch pb_batch;

/* natoms[nsys] atoms per system; flags as pb_md_create. */
int pb_batch_create(const uint32_t *natoms, uint32_t nsys, uint32_t flags, pb_batch **out);
/* A new batch whose system k continues system src[k] of `old` (state,
 * box, LJ table, dt, kB and the Gaussian friction carried over bit for bit)
 * or, when src[k] < 0, is a new system of natoms[k] atoms to be set up with
 * pb_batch_set_system and pb_batch_import.  natoms[k] is ignored when
 * src[k] >= 0.  Call pb_batch_setup_cells before stepping. */
int pb_batch_repack(const pb_batch *old, const int32_t *src, const uint32_t *natoms, uint32_t nsys,
                    pb_batch **out);
int pb_batch_destroy(pb_batch *b);
int pb_batch_set_stream(pb_batch *b, void *stream);
const char *pb_batch_last_error(const pb_batch *b);
/* *nsys systems, *natoms_total atoms; atom0 (optional, nsys + 1 entries):
 * first packed atom of every system. */
int pb_batch_size(const pb_batch *b, uint32_t *nsys, uint32_t *natoms_total, uint32_t *atom0);
/* Box, LJ cutoff (rmax2 = rc^2), LJ (sigma, epsilon) per ordered type pair,
 * time step and kB of system `sys` (setCell, rmax2, setLJparams of one
 * system). */
int pb_batch_set_system(pb_batch *b, uint32_t sys, const float cell6[6], float rc,
                        const float *sigma_eps, uint32_t ntypes, float dt, float kB);
/* Per-pair cutoffs for system `sys` (pb_md_set_lj_cut): (sigma, epsilon, rc)
 * per ordered type pair, after pb_batch_set_system. */
int pb_batch_set_lj_cut(pb_batch *b, uint32_t sys, const float *sigma_eps_rc, uint32_t ntypes);
/* As pb_md_import_arrays, for system `sys`. */
int pb_batch_import(pb_batch *b, uint32_t sys, const double *r3, const double *v3,
                    const double *mass, const uint32_t *type);
/* Cell grids of all systems; rmax[sys] per system, or NULL for each system's
 * LJ cutoff.  Also uploads the parameters given to pb_batch_set_system and
 * pb_batch_set_lj_cut since the last setup (they take effect here). */
int pb_batch_setup_cells(pb_batch *b, const float *rmax);
/* Cell build + force for all systems (pb_md_build_cells + pb_md_force). */
int pb_batch_force(pb_batch *b, uint32_t flags);
int pb_batch_clear_force(pb_batch *b);
/* `steps` whole steps of every system (pb_md_run), each with its own dt. */
int pb_batch_run(pb_batch *b, int mode, uint32_t steps);
int pb_batch_run_timed(pb_batch *b, int mode, uint32_t steps, float *ms);
int pb_batch_profile(pb_batch *b, int mode, uint32_t steps, double ms[3]);
/* Step budgets: system s runs steps[s] more time steps and then stays as it
 * is while the others go on (its cells are still binned, but no force or
 * integration work is done for it), so systems with different step counts
 * share one graph replay and each ends after exactly its own count.  NULL
 * removes the budgets.  pb_batch_get_steps_left reads the counters back. */
int pb_batch_set_steps_left(pb_batch *b, const uint32_t *steps);
int pb_batch_get_steps_left(pb_batch *b, uint32_t *steps);
/* Per-system sums (out[nsys]), temperatures (T[nsys]), status words
 * (bits[nsys], cleared by the call). */
int pb_batch_reduce(pb_batch *b, pb_md_sums *out);
int pb_batch_temperature(pb_batch *b, double *T);
int pb_batch_status(pb_batch *b, uint32_t *bits);
/* Per-system factors / v1 values (nsys doubles each). */
int pb_batch_scale_velocities(pb_batch *b, const double *s);
int pb_batch_adjust_velocities(pb_batch *b, const double *v1);
/* Per-atom fields R, V, VD, F, FOLD, MINV, TYPE, MASS of system `sys`
 * (sizes as pb_md_get for that system's atom count). */
int pb_batch_get(pb_batch *b, uint32_t sys, int field, void *host, size_t bytes);
int pb_batch_set(pb_batch *b, uint32_t sys, int field, const void *host, size_t bytes);
/* Launch parameters of the force kernel, chosen by the caller or an
 * autotuner: threads per CTA (128 or 256), and a scale for the z-run length
 * of every work item (1.0 = default; forces do not depend on either).  Takes
 * effect at the next pb_batch_setup_cells. */
int pb_batch_set_tuning(pb_batch *b, int force_threads, float seg_scale);
/* Bytes of device memory a batch of these systems holds after setup_cells
 * (estimate from the atom counts and grids; used for admission control). */
int pb_batch_estimate_bytes(const uint32_t *natoms, const float *cells6, const float *rmax,
                            uint32_t nsys, uint32_t flags, size_t *bytes);

/* ---- serving: a request loop over the batch ---------------------------------
 *
 * No counterpart in the reference.  A pb_srv owns a scheduler thread and one
 * resident pb_batch.  Submitted MD jobs wait in a FIFO queue until the
 * memory estimate of the resident set plus the job fits the HBM budget; the
 * scheduler then packs them into the batch at the next chunk boundary, where
 * finished jobs also leave (their final state is copied to host memory).
 * Between boundaries the batch advances by whole graph-replayed steps, every
 * job under its own step budget, so each job ends after exactly its step
 * count, with the result it would have alone (bit for bit, same flags). */
typedef struct pb_srv pb_srv;

/* The library's device memory pool: every handle allocates from it, and it
   keeps the memory they free.  Growing it maps new pages, which inside a busy
   process took up to a second per growth.  pb_pool_reserve takes `bytes` into
   it at once (PB_ERR_OOM when they are not free); pb_pool_trim hands its unused
   memory back to the device.  No counterpart in the reference. */
int pb_pool_reserve(size_t bytes);
int pb_pool_trim(void);

typedef struct pb_srv_config {
  size_t hbm_budget;      /* bytes the resident batch may hold (estimate); 0 = 90% of free */
  uint64_t max_atoms;     /* resident atom cap (0 = none): bounds the step time */
  uint32_t max_jobs;      /* resident job cap (0 = none) */
  float chunk_ms;         /* target GPU time between chunk boundaries (0 = 100 ms) */
  uint32_t flags;         /* PB_MD_VEL_FP64 | PB_MD_ACC_FP64 */
  int mode;               /* PB_MODE_VV or PB_MODE_GAUSS */
  int force_threads;      /* 0 = default (256) */
  float seg_scale;        /* 0 = 1.0 */
  size_t reserve_bytes;   /* device memory taken into the library's pool at creation
                             (pb_pool_reserve), so that repacks never wait for the pool
                             to grow; pb_srv_destroy then trims the pool (pb_pool_trim),
                             which hands back the unused memory of every handle.
                             0 = none, SIZE_MAX = the whole HBM budget.  Not available:
                             the server runs without it. */
} pb_srv_config;

typedef struct pb_srv_job {
  uint32_t natoms;
  float cell6[6];
  float rc;                   /* LJ cutoff (and cell size) */
  const float *sigma_eps;     /* (sigma, epsilon) per ordered type pair */
  const float *sigma_eps_rc;  /* optional per-pair cutoffs (sigma, epsilon, rc), or NULL */
  uint32_t ntypes;
  float dt, kB;
  uint32_t steps;
  const double *r3, *v3, *mass;  /* host arrays, copied by pb_srv_submit; v3/mass may be NULL */
  const uint32_t *type;          /* or NULL */
} pb_srv_job;

#define PB_JOB_QUEUED 0
#define PB_JOB_RUNNING 1
#define PB_JOB_DONE 2
#define PB_JOB_FAILED 3

typedef struct pb_srv_job_info {
  uint64_t id;
  int state;
  uint32_t natoms, steps;
  double t_submit, t_admit, t_done;  /* seconds on the server clock (pb_srv_now) */
  uint32_t device_status;            /* status bits the kernels raised for this job */
} pb_srv_job_info;

typedef struct pb_srv_stats {
  uint64_t submitted, done, failed, rejected;
  double atom_steps;          /* completed atom-steps of finished jobs */
  double gpu_seconds;         /* device time of the step chunks (CUDA events) */
  double repack_seconds;      /* host time spent repacking at chunk boundaries */
  uint64_t chunks, repacks;
  uint64_t peak_jobs, peak_atoms;
  size_t peak_bytes;          /* largest resident-set memory estimate */
} pb_srv_stats;

int pb_srv_create(const pb_srv_config *cfg, pb_srv **out);
/* Stops the scheduler (running jobs are abandoned) and frees everything. */
int pb_srv_destroy(pb_srv *s);
/* Queue a job; its arrays are copied before the call returns.  A job whose
 * own memory estimate exceeds the budget is rejected (PB_ERR_OOM). */
int pb_srv_submit(pb_srv *s, const pb_srv_job *job, uint64_t *id);
/* Block until job `id` is done or failed (timeout_s < 0: no limit). */
int pb_srv_wait(pb_srv *s, uint64_t id, double timeout_s);
/* Block until every submitted job is done or failed. */
int pb_srv_drain(pb_srv *s, double timeout_s);
/* Ids of jobs finished since the last poll (up to max). */
int pb_srv_poll(pb_srv *s, uint64_t *ids, uint32_t max, uint32_t *n);
int pb_srv_info(pb_srv *s, uint64_t id, pb_srv_job_info *info);
/* Final state of a finished job: r4 float4[n] positions, v velocities
 * (float4[n] or double[3n] planes with PB_MD_VEL_FP64, vbytes to match),
 * F4 float4[n] last forces; any pointer may be NULL. */
int pb_srv_result(pb_srv *s, uint64_t id, void *r4, void *v, size_t vbytes, void *F4);
/* Forget a finished job and its stored result. */
int pb_srv_release(pb_srv *s, uint64_t id);
int pb_srv_stats_get(pb_srv *s, pb_srv_stats *st);
double pb_srv_now(const pb_srv *s);
const char *pb_srv_last_error(const pb_srv *s);

/* Library version string. */
const char *pb_version(void);

#ifdef __cplusplus
}
#endif

#endif /* PB_PB_H */
