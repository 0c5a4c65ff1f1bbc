// Host engine shared by the single-system handle (pb_md, one system) and the
// batch handle (pb_batch, many packed systems): device buffers, the cell
// plan, kernel launch sequences and CUDA-graph replay of whole steps.
#pragma once

#include <string>
#include <vector>

#include "integrate.cuh"
#include "md.cuh"

namespace pb {

// Host-side parameters of one system.
struct SysParams {
  uint32_t n = 0;
  float cell[6] = {0, 1, 0, 1, 0, 1};
  bool cell_set = false;
  float rmax = 0.f, rmax2 = 0.f, kB = 1.f;
  LJTable lj{};
  bool lj_set = false, lj_percut = false;
  Grid grid{};
  int seg = 1;
  uint32_t cap = 0;
  uint32_t cap_half = 0;  // stage capacity of the half-shell force kernel
  double m0 = 1.0;
  float dt = 0.005f;
  bool r_set = false;     // positions imported or set (the cell build may be timed)
  bool periodic = true;   // false: open boundaries (pb_md_setup_cells(periodic = 0))
  std::vector<uint32_t> key_of_ref, ref_of_key;  // reference cell id <-> packed key - cell0
};

struct Engine {
  std::string err;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  uint32_t flags = 0;  // PB_MD_VEL_FP64 | PB_MD_ACC_FP64
  uint32_t nsys = 0, N = 0;
  std::vector<SysParams> sp;
  std::vector<uint32_t> atom0;  // first atom of each system (+ total)
  std::vector<SysInt> sysint;   // host mirror of d_sysint
  int force_threads = 256;
  float seg_scale = 1.f;  // z-run length scale of the force work items

  // per-atom state
  float4 *r = nullptr, *v = nullptr, *F[2] = {nullptr, nullptr};
  int cur = 0;   // the next force call writes F[cur]; the next step uses F[1 - cur] as Fold
  int last = 0;  // F[last] holds the most recent force (reference field F)
  double *vd = nullptr;
  float *minv = nullptr, *mass = nullptr;
  uint16_t *type = nullptr;
  uint32_t *sysid = nullptr;  // only with nsys > 1

  // integration
  SysInt *d_sysint = nullptr;
  BlockMap *d_map = nullptr;
  uint32_t nblocks = 0;
  double *ipartials = nullptr;
  DevScalars *sc = nullptr;
  uint32_t *status = nullptr;
  double *d_fac = nullptr;  // per-system factors for scale / adjust
  double *h_read = nullptr;  // pinned host word for per-step scalar reads (lazy)
  LJTable *d_lj = nullptr;

  // cell list (after setup_cells)
  bool cells_ready = false;
  uint32_t ncells = 0;
  uint32_t *key = nullptr, *within = nullptr, *tilesum = nullptr, *count = nullptr,
           *start = nullptr, *pid_tmp = nullptr,
           *pid = nullptr, *slot = nullptr, *colrank = nullptr, *colxy = nullptr,
           *d_item0 = nullptr;
  // cell buckets of the two-kernel build: bucket_cap ids per cell, the
  // overflow list, tile counts, and two control words
  uint32_t *bucket = nullptr, *tcount = nullptr, *cctl = nullptr;
  uint2 *ovf = nullptr;
  uint32_t bucket_cap = 0, ntile = 0, tile_atoms = 0;
  // which cell build the steps use: the bucket build (true) or the six-kernel
  // counting sort; chosen by timing both at cell set-up (same result bits)
  bool cells_bucket = true;
  bool cells_chosen = false;  // set: keep cells_bucket at the next set-up (repacks)
  float4 *rs = nullptr;
  float *xs = nullptr, *ys = nullptr, *zs = nullptr;  // SoA mirrors of rs
  uint32_t *ts = nullptr;
  uint32_t mirrorN = 0;
  SysDesc *d_sys = nullptr;
  ForceItem *d_items = nullptr;
  uint32_t nitems = 0;
  std::vector<uint32_t> item0, cell0;
  double *fpartials = nullptr;
  uint32_t *fqueue = nullptr;  // the force kernel's item counter
  uint32_t cap_max = 0;
  uint32_t cap_half_max = 0;
  unsigned long long *facc = nullptr;  // half-shell force sums: fine and coarse, 2 x 3 x N
  uint32_t force_test_flags = 0;       // ForceBufs::test_flags of the next force call
  uint32_t force_wait_polls = 0;       // ForceBufs::wait_polls of the next force call
  bool energy_valid = false;
  bool mv2_fresh = false;  // sc.mv2 holds sum m v^2 of the current velocities

  // Verlet neighbour list (single-system handles; see nlist.cu): while on,
  // force calls use the list and whole steps skip the cell-list build
  bool nl_on = false, nl_built = false;
  float nl_skin = 0.f;
  uint32_t nl_cap = 0;  // entries per row
  uint32_t *nl_idx = nullptr, *nl_cnt = nullptr, *nl_atom = nullptr, *nl_max = nullptr;
  float4 *nl_r0 = nullptr, *nl_rl = nullptr;
  double *nl_partials = nullptr;
  uint32_t *d_nl_item0 = nullptr;  // {0, blocks}: the list force's energy partials

  // per-system step budgets (serving): device counters, nullptr = no limits
  uint32_t *steps_left = nullptr;
  uint64_t steps_done = 0;           // time steps issued since creation
  std::vector<uint64_t> budget_set;  // steps_done when each budget was set
  std::vector<uint64_t> budget_end;  // steps_done at which each budget runs out
  std::vector<int> last_at_set;      // `last` when each budget was set

  // CUDA graphs of two whole steps and of one step, each for both parities of
  // the F ping-pong: a captured step bakes in which buffer is F and which is
  // Fold, so a graph only replays at the parity it was captured at
  cudaGraphExec_t graph2[2] = {nullptr, nullptr};
  cudaGraphExec_t graph1[2] = {nullptr, nullptr};
  int graph_mode = -1;
  std::vector<float> graph_dt;
};

// All return pb_status codes; on failure e.err says why.
// zero_state = false leaves r, v, F and type unwritten: a repack's gather
// writes every atom of them (continuing systems copied, new ones zeroed).
int engine_init(Engine &e, const uint32_t *natoms, uint32_t nsys, uint32_t flags,
                bool zero_state = true);
void engine_free(Engine &e);
int engine_set_stream(Engine &e, cudaStream_t s);
int engine_upload_lj(Engine &e);
int engine_upload_sysint(Engine &e);
int engine_import(Engine &e, uint32_t sys, const double *r3, const double *v3, const double *mass,
                  const uint32_t *type);
int engine_setup_cells(Engine &e);
bool engine_ready(const Engine &e);

int engine_build(Engine &e);
int engine_force(Engine &e, bool energy);
int engine_evolve(Engine &e, int mode, int wrap);
int engine_wrap(Engine &e);
int engine_step(Engine &e, int mode);
// Device scratch from the engine's pool, on its stream (stream-ordered).
cudaError_t engine_alloc_bytes(Engine &e, void **p, size_t bytes);
void engine_free_bytes(Engine &e, void *p);
// The device pool engines allocate from: reserve takes `bytes` into it at once
// (PB_ERR_OOM when they are not free); trim hands its unused memory back.
int engine_pool_reserve(size_t bytes);
void engine_pool_trim();
// Neighbour list: thickness >= 0 turns it on (rows within rc + thickness),
// thickness < 0 off; make rebuilds the cell list and the neighbour list.
int engine_use_nlist(Engine &e, float thickness);
int engine_make_nlist(Engine &e);
// Mean and largest row length of the last build, and the row capacity.
int engine_nlist_info(Engine &e, double out[3]);
// Pair counts per distance bin of the current positions (single system);
// *rnum = the bin count of the reference's rule; counts (host) when non-null.
int engine_gr(Engine &e, float rstep, float rmax, uint64_t *counts, uint32_t *rnum);
int engine_run(Engine &e, int mode, uint32_t steps);
int engine_profile(Engine &e, int mode, uint32_t steps, double ms[3]);
int engine_clear_force(Engine &e);
int engine_mv2(Engine &e);
int engine_fv(Engine &e);
int engine_scale(Engine &e, const double *factors);
int engine_adjust(Engine &e, const double *v1);
int engine_correct_force(Engine &e, const double *lambda);
// Soft-core force (initialAnnealing) into the force buffer, cells as built.
int engine_force_softcore(Engine &e, float rc, float f0);
// Euler step with the latest force: r += v dt, v += F/m dt, wrap.
int engine_euler(Engine &e, float dt);
// Steepest-descent relaxation: iters x (cell build, relaxation force, move).
int engine_minimize(Engine &e, uint32_t iters, float alpha, float max_disp);
int engine_set_xi(Engine &e, const double *xi);
int engine_scalars(Engine &e, std::vector<DevScalars> &out);
int engine_status(Engine &e, std::vector<uint32_t> &bits);
void engine_drop_graph(Engine &e);
void engine_set_dt(Engine &e, float dt);
// Step budgets: system s runs steps[s] more steps, then its state stays as it
// is (the force and integration kernels skip it).  steps == nullptr removes
// all limits.
int engine_set_steps_left(Engine &e, const uint32_t *steps);
int engine_get_steps_left(Engine &e, uint32_t *steps);
// Index of the force buffer holding system s's most recent force.
int engine_force_buffer(const Engine &e, uint32_t s);
// True once system s has used up its step budget.
bool engine_finished(const Engine &e, uint32_t s);

// LJ table of one system from (sigma, epsilon[, rc]) per ordered type pair
// (stride 2 or 3), as _setLJparams (kernelinline.hh:120-134) stores it:
// sigma^2 and 24 epsilon, plus the shift of the potential at the cutoff.
void lj_table_fill(SysParams &P, const float *p, uint32_t nt, int stride, bool percut);
// Common cutoff rmax2 for a table filled without per-pair cutoffs.
void lj_table_set_rmax2(SysParams &P, float rmax2);

IntegrateArgs engine_iargs(Engine &e, int wrap);
CellBufs engine_cbufs(Engine &e);
ForceBufs engine_fbufs(Engine &e);

}  // namespace pb
