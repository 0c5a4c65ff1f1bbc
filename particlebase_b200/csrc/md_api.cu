// Host implementation of the single-system C ABI (include/pb/pb.h).  A pb_md
// handle is the engine with one system; the batch API (batch_api.cu) drives
// the same engine with many.
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/pb/pb.h"
#include "engine.h"
#include "plan.h"

using namespace pb;

static_assert(sizeof(pb_particle) == 96, "pb_particle must match ParticleBase");
static_assert(PB_STATUS_SMEM_OVERFLOW == pb::kStatusSmemOverflow &&
                  PB_STATUS_NONFINITE == pb::kStatusNonFinite &&
                  PB_STATUS_WAIT_TIMEOUT == pb::kStatusWaitTimeout &&
                  PB_STATUS_CELL_OVERFLOW == pb::kStatusCellOverflow &&
                  PB_STATUS_NOCONVERGE == pb::kStatusNoConverge &&
                  PB_STATUS_NLIST_OVERFLOW == pb::kStatusNlistOverflow &&
                  PB_STATUS_STALE_NLIST == pb::kStatusStaleList,
              "status bits of the C ABI and the kernels");
static_assert(offsetof(pb_particle, is_fixed) == 56, "pb_particle layout");
static_assert(offsetof(pb_particle, a) == 64, "pb_particle layout");
static_assert(offsetof(pb_particle, type) == 88, "pb_particle layout");

struct pb_md {
  Engine e;
  SysParams &p() { return e.sp[0]; }
  const SysParams &p() const { return e.sp[0]; }
};

namespace {

int fail(pb_md *h, int code, const std::string &msg) {
  if (h) h->e.err = msg;
  return code;
}

#define H_CUDA(call)                                                                   \
  do {                                                                                 \
    cudaError_t c_ = (call);                                                           \
    if (c_ != cudaSuccess)                                                             \
      return fail(h, PB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(c_)); \
  } while (0)

}  // namespace

extern "C" {

const char *pb_version(void) { return "particlebase_b200 0.2 (sm_100a)"; }

int pb_plan_grid(const float cell6[6], float rmax, uint32_t n3[3], float len3[3]) {
  if (!cell6 || !n3 || !len3) return PB_ERR_ARG;
  Grid g;
  if (!make_grid(cell6, rmax, g)) return PB_ERR_ARG;
  for (int k = 0; k < 3; ++k) {
    n3[k] = (uint32_t)g.n[k];
    len3[k] = g.len[k];
  }
  return PB_OK;
}

int pb_plan_columns(uint32_t nx, uint32_t ny, uint32_t *rank) {
  if (!rank || nx == 0 || ny == 0) return PB_ERR_ARG;
  std::vector<uint32_t> r, xy;
  morton_columns((int)nx, (int)ny, r, xy);
  std::memcpy(rank, r.data(), sizeof(uint32_t) * r.size());
  return PB_OK;
}

int pb_md_create(uint32_t n, uint32_t flags, pb_md **out) {
  if (!out || n == 0) return PB_ERR_ARG;
  *out = nullptr;
  pb_md *h = new pb_md;
  const int rc = engine_init(h->e, &n, 1, flags);
  if (rc) {
    engine_free(h->e);
    delete h;
    return rc;
  }
  *out = h;
  return PB_OK;
}

int pb_md_destroy(pb_md *h) {
  if (!h) return PB_ERR_ARG;
  engine_free(h->e);
  delete h;
  return PB_OK;
}

int pb_md_set_stream(pb_md *h, void *stream) {
  if (!h) return PB_ERR_ARG;
  return engine_set_stream(h->e, (cudaStream_t)stream);
}

const char *pb_md_last_error(const pb_md *h) { return h ? h->e.err.c_str() : "null handle"; }

int pb_md_status(pb_md *h, uint32_t *bits) {
  if (!h || !bits) return PB_ERR_ARG;
  std::vector<uint32_t> b;
  const int rc = engine_status(h->e, b);
  if (rc) return rc;
  *bits = b[0];
  return PB_OK;
}

int pb_md_set_cell(pb_md *h, const float cell6[6]) {
  if (!h || !cell6) return PB_ERR_ARG;
  for (int k = 0; k < 3; ++k)
    if (!(cell6[2 * k + 1] > cell6[2 * k])) return fail(h, PB_ERR_ARG, "empty box");
  std::memcpy(h->p().cell, cell6, sizeof(float) * 6);
  h->p().cell_set = true;
  h->e.cells_ready = false;  // the grid depends on the box: setup_cells again
  engine_drop_graph(h->e);
  return engine_upload_sysint(h->e);
}

int pb_md_set_lj(pb_md *h, const float *sigma_eps, uint32_t ntypes) {
  if (!h || !sigma_eps || ntypes < 1 || ntypes > (uint32_t)kMaxTypes) return PB_ERR_ARG;
  lj_table_fill(h->p(), sigma_eps, ntypes, 2, false);
  engine_drop_graph(h->e);
  return engine_upload_lj(h->e);
}

int pb_md_set_lj_cut(pb_md *h, const float *p, uint32_t ntypes) {
  if (!h || !p || ntypes < 1 || ntypes > (uint32_t)kMaxTypes) return PB_ERR_ARG;
  lj_table_fill(h->p(), p, ntypes, 3, true);
  engine_drop_graph(h->e);
  return engine_upload_lj(h->e);
}

int pb_md_set_rmax2(pb_md *h, float rmax2) {
  if (!h || !(rmax2 > 0)) return PB_ERR_ARG;
  lj_table_set_rmax2(h->p(), rmax2);
  if (!h->p().lj_set) return PB_OK;
  engine_drop_graph(h->e);
  return engine_upload_lj(h->e);
}

int pb_md_set_kB(pb_md *h, float kB) {
  if (!h || !(kB > 0)) return PB_ERR_ARG;
  h->p().kB = kB;
  return PB_OK;
}

int pb_md_import_arrays(pb_md *h, const double *r3, const double *v3, const double *mass,
                        const uint32_t *type) {
  if (!h || !r3) return PB_ERR_ARG;
  return engine_import(h->e, 0, r3, v3, mass, type);
}

int pb_md_import(pb_md *h, const pb_particle *p, uint32_t n) {
  if (!h || !p || n != h->e.N) return PB_ERR_ARG;
  std::vector<double> r3(3 * (size_t)n), v3(3 * (size_t)n), m(n);
  std::vector<uint32_t> t(n);
  for (uint32_t i = 0; i < n; ++i) {
    for (int k = 0; k < 3; ++k) {
      r3[3 * i + k] = p[i].r[k];
      v3[3 * i + k] = p[i].v[k];
    }
    m[i] = p[i].m;
    t[i] = p[i].type;
  }
  return pb_md_import_arrays(h, r3.data(), v3.data(), m.data(), t.data());
}

int pb_md_setup_cells(pb_md *h, float rmax, int periodic) {
  if (!h || !(rmax > 0)) return PB_ERR_ARG;
  if (!h->p().cell_set) return fail(h, PB_ERR_STATE, "set the cell first");
  h->p().rmax = rmax;
  h->p().periodic = periodic != 0;
  return engine_setup_cells(h->e);
}

int pb_md_grid(const pb_md *h, uint32_t n3[3], float len3[3], uint32_t *ncells) {
  if (!h || !h->e.cells_ready) return PB_ERR_STATE;
  const Grid &g = h->p().grid;
  for (int k = 0; k < 3; ++k) {
    if (n3) n3[k] = (uint32_t)g.n[k];
    if (len3) len3[k] = g.len[k];
  }
  if (ncells) *ncells = g.ncells;
  return PB_OK;
}

int pb_md_build_cells(pb_md *h) { return h ? engine_build(h->e) : PB_ERR_ARG; }

int pb_md_use_nlist(pb_md *h, float thickness) {
  return h ? engine_use_nlist(h->e, thickness) : PB_ERR_ARG;
}

int pb_md_make_nlist(pb_md *h) { return h ? engine_make_nlist(h->e) : PB_ERR_ARG; }

int pb_md_nlist_info(pb_md *h, double out[3]) {
  if (!h || !out) return PB_ERR_ARG;
  return engine_nlist_info(h->e, out);
}

int pb_md_gr(pb_md *h, float rstep, float rmax, uint64_t *counts, uint32_t *rnum) {
  return h ? engine_gr(h->e, rstep, rmax, counts, rnum) : PB_ERR_ARG;
}

int pb_md_force(pb_md *h, uint32_t flags) {
  return h ? engine_force(h->e, (flags & PB_FORCE_ENERGY) != 0) : PB_ERR_ARG;
}

int pb_md_force_wait_test(pb_md *h, uint32_t polls) {
  if (!h || polls == 0) return PB_ERR_ARG;
  h->e.force_test_flags = 1u;
  h->e.force_wait_polls = polls;
  const int rc = engine_force(h->e, false);
  h->e.force_test_flags = 0u;
  h->e.force_wait_polls = 0u;
  if (rc) return rc;
  return cudaStreamSynchronize(h->e.stream) == cudaSuccess ? PB_OK : PB_ERR_CUDA;
}

int pb_md_clear_force(pb_md *h) { return h ? engine_clear_force(h->e) : PB_ERR_ARG; }

int pb_md_step_vv(pb_md *h, float dt) {
  if (!h) return PB_ERR_ARG;
  engine_set_dt(h->e, dt);
  return engine_evolve(h->e, PB_MODE_VV, 0);
}

int pb_md_step_gauss(pb_md *h, float dt, double tol) {
  (void)tol;  // the friction is solved in closed form
  if (!h) return PB_ERR_ARG;
  engine_set_dt(h->e, dt);
  return engine_evolve(h->e, PB_MODE_GAUSS, 0);
}

int pb_md_wrap(pb_md *h) { return h ? engine_wrap(h->e) : PB_ERR_ARG; }

int pb_md_run(pb_md *h, float dt, int mode, uint32_t steps) {
  if (!h) return PB_ERR_ARG;
  engine_set_dt(h->e, dt);
  return engine_run(h->e, mode, steps);
}

int pb_md_run_timed(pb_md *h, float dt, int mode, uint32_t steps, float *ms) {
  if (!h || !ms) return PB_ERR_ARG;
  engine_set_dt(h->e, dt);
  cudaEvent_t a, b;
  H_CUDA(cudaEventCreate(&a));
  H_CUDA(cudaEventCreate(&b));
  H_CUDA(cudaEventRecord(a, h->e.stream));
  const int rc = engine_run(h->e, mode, steps);
  cudaEventRecord(b, h->e.stream);
  cudaEventSynchronize(b);
  cudaEventElapsedTime(ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return rc;
}

int pb_md_profile(pb_md *h, float dt, int mode, uint32_t steps, double ms[3]) {
  if (!h || !ms || steps == 0) return PB_ERR_ARG;
  engine_set_dt(h->e, dt);
  return engine_profile(h->e, mode, steps, ms);
}

int pb_md_cell_build_kernels(pb_md *h, uint32_t *kernels) {
  if (!h || !kernels) return PB_ERR_ARG;
  if (!h->e.cells_ready) return fail(h, PB_ERR_STATE, "setup_cells first");
  *kernels = h->e.cells_bucket ? 2u : 6u;
  return PB_OK;
}

int pb_md_pair_stats(pb_md *h, double out[2]) {
  if (!h || !out || !h->e.cells_ready) return PB_ERR_STATE;
  Engine &e = h->e;
  const SysParams &P = h->p();
  const uint32_t C = P.grid.ncells;
  std::vector<uint32_t> start(C + 1);
  H_CUDA(cudaMemcpyAsync(start.data(), e.start, 4 * (size_t)(C + 1), cudaMemcpyDeviceToHost,
                         e.stream));
  std::vector<DevScalars> sc;
  const int rc = engine_scalars(e, sc);
  if (rc) return rc;
  std::vector<uint32_t> nb;
  neighbor_table(P.grid, nb);
  double cand = 0;
  for (uint32_t ref = 0; ref < C; ++ref) {
    const uint32_t k = P.key_of_ref[ref];
    const double nc = start[k + 1] - start[k];
    double around = 0;
    for (int j = 0; j < 27; ++j) {
      const uint32_t kn = P.key_of_ref[nb[(size_t)ref * 27 + j]];
      around += start[kn + 1] - start[kn];
    }
    cand += nc * (around - 1.0);
  }
  out[0] = cand;
  out[1] = e.energy_valid ? sc[0].npairs : NAN;
  return PB_OK;
}

int pb_md_reduce(pb_md *h, pb_md_sums *out) {
  if (!h || !out) return PB_ERR_ARG;
  int rc = engine_mv2(h->e);
  if (!rc) rc = engine_fv(h->e);
  std::vector<DevScalars> sc;
  if (!rc) rc = engine_scalars(h->e, sc);
  if (rc) return rc;
  out->mv2 = sc[0].mv2;
  out->fv = sc[0].fv;
  out->pe = h->e.energy_valid ? sc[0].pe : NAN;
  out->pe_shift = h->e.energy_valid ? sc[0].pe_shift : NAN;
  out->virial = h->e.energy_valid ? sc[0].virial : NAN;
  out->xi = sc[0].xi_old;
  return PB_OK;
}

int pb_md_temperature(pb_md *h, double *T) {
  if (!h || !T) return PB_ERR_ARG;
  if (!h->e.mv2_fresh) {  // otherwise the last step's sum is still current
    const int rc = engine_mv2(h->e);
    if (rc) return rc;
  }
  // a pinned word: the driver loop reads the temperature every step, and a
  // copy to pageable memory goes through a staging buffer
  if (!h->e.h_read) H_CUDA(cudaMallocHost(&h->e.h_read, sizeof(double)));
  H_CUDA(cudaMemcpyAsync(h->e.h_read, &h->e.sc[0].mv2, sizeof(double), cudaMemcpyDeviceToHost,
                         h->e.stream));
  H_CUDA(cudaStreamSynchronize(h->e.stream));
  *T = *h->e.h_read / (3.0 * h->e.N * h->p().kB);
  return PB_OK;
}

int pb_md_scale_velocities(pb_md *h, double s) { return h ? engine_scale(h->e, &s) : PB_ERR_ARG; }

int pb_md_adjust_velocities(pb_md *h, double v1) {
  return h ? engine_adjust(h->e, &v1) : PB_ERR_ARG;
}

int pb_md_correct_force(pb_md *h, double lambda) {
  return h ? engine_correct_force(h->e, &lambda) : PB_ERR_ARG;
}

int pb_md_force_softcore(pb_md *h, float rc, float f0) {
  return h ? engine_force_softcore(h->e, rc, f0) : PB_ERR_ARG;
}

int pb_md_step_euler(pb_md *h, float dt) { return h ? engine_euler(h->e, dt) : PB_ERR_ARG; }

int pb_md_minimize(pb_md *h, uint32_t iters, float alpha, float max_disp) {
  return h ? engine_minimize(h->e, iters, alpha, max_disp) : PB_ERR_ARG;
}

int pb_md_set_xi(pb_md *h, double xi) { return h ? engine_set_xi(h->e, &xi) : PB_ERR_ARG; }

int pb_md_mean_mass(const pb_md *h, double *m0) {
  if (!h || !m0) return PB_ERR_ARG;
  *m0 = h->p().m0;
  return PB_OK;
}

int pb_md_size(const pb_md *h, uint32_t *n) {
  if (!h || !n) return PB_ERR_ARG;
  *n = h->e.N;
  return PB_OK;
}

int pb_md_field_bytes(const pb_md *h, int field, size_t *bytes) {
  if (!h || !bytes) return PB_ERR_ARG;
  const size_t N = h->e.N, C = h->e.cells_ready ? h->p().grid.ncells : 0;
  switch (field) {
    case PB_FIELD_R: case PB_FIELD_V: case PB_FIELD_F: case PB_FIELD_FOLD: case PB_FIELD_R_SORTED:
      *bytes = 16 * N; break;
    case PB_FIELD_VD: *bytes = 24 * N; break;
    case PB_FIELD_MINV: case PB_FIELD_MASS: case PB_FIELD_CELL_OF: case PB_FIELD_PID:
      *bytes = 4 * N; break;
    case PB_FIELD_TYPE: *bytes = 2 * N; break;
    case PB_FIELD_CELL_START: *bytes = 4 * (C + 1); break;
    case PB_FIELD_CELL_KEY: *bytes = 4 * C; break;
    case PB_FIELD_NEIGHBORS: *bytes = 4 * 27 * C; break;
    default: return PB_ERR_NOTFOUND;
  }
  return PB_OK;
}

int pb_md_get(pb_md *h, int field, void *host, size_t bytes) {
  if (!h || !host) return PB_ERR_ARG;
  Engine &e = h->e;
  size_t need = 0;
  const int rc = pb_md_field_bytes(h, field, &need);
  if (rc) return rc;
  const bool cell_field = field >= PB_FIELD_CELL_OF && field <= PB_FIELD_R_SORTED;
  if (cell_field && !e.cells_ready) return fail(h, PB_ERR_STATE, "no cell list");
  if (bytes != need) return fail(h, PB_ERR_ARG, "size mismatch for field");
  const void *src = nullptr;
  switch (field) {
    case PB_FIELD_R: src = e.r; break;
    case PB_FIELD_V:
      if (!e.v) return fail(h, PB_ERR_STATE, "handle keeps FP64 velocities");
      src = e.v; break;
    case PB_FIELD_VD:
      if (!e.vd) return fail(h, PB_ERR_STATE, "handle keeps FP32 velocities");
      src = e.vd; break;
    case PB_FIELD_F: src = e.F[engine_force_buffer(e, 0)]; break;
    case PB_FIELD_FOLD: src = e.F[1 - e.cur]; break;
    case PB_FIELD_MINV: src = e.minv; break;
    case PB_FIELD_MASS: src = e.mass; break;
    case PB_FIELD_TYPE: src = e.type; break;
    case PB_FIELD_PID: src = e.pid; break;
    case PB_FIELD_CELL_START: src = e.start; break;
    case PB_FIELD_R_SORTED: src = e.rs; break;
    case PB_FIELD_CELL_OF: {
      std::vector<uint32_t> k(e.N);
      H_CUDA(cudaMemcpyAsync(k.data(), e.key, 4 * (size_t)e.N, cudaMemcpyDeviceToHost, e.stream));
      H_CUDA(cudaStreamSynchronize(e.stream));
      uint32_t *o = (uint32_t *)host;
      for (uint32_t i = 0; i < e.N; ++i) o[i] = h->p().ref_of_key[k[i]];
      return PB_OK;
    }
    case PB_FIELD_CELL_KEY:
      std::memcpy(host, h->p().key_of_ref.data(), need);
      return PB_OK;
    case PB_FIELD_NEIGHBORS: {
      std::vector<uint32_t> t;
      neighbor_table(h->p().grid, t);
      std::memcpy(host, t.data(), need);
      return PB_OK;
    }
    default: return PB_ERR_NOTFOUND;
  }
  H_CUDA(cudaMemcpyAsync(host, src, need, cudaMemcpyDeviceToHost, e.stream));
  H_CUDA(cudaStreamSynchronize(e.stream));
  return PB_OK;
}

int pb_md_set(pb_md *h, int field, const void *host, size_t bytes) {
  if (!h || !host) return PB_ERR_ARG;
  Engine &e = h->e;
  size_t need = 0;
  const int rc = pb_md_field_bytes(h, field, &need);
  if (rc) return rc;
  if (bytes != need) return fail(h, PB_ERR_ARG, "size mismatch for field");
  e.mv2_fresh = false;  // velocities or masses may change
  void *dst = nullptr;
  switch (field) {
    case PB_FIELD_R:
      dst = e.r;
      for (auto &P : e.sp) P.r_set = true;
      break;
    case PB_FIELD_V: dst = e.v; break;
    case PB_FIELD_VD: dst = e.vd; break;
    case PB_FIELD_F: dst = e.F[e.last]; break;
    case PB_FIELD_FOLD: dst = e.F[1 - e.cur]; break;
    case PB_FIELD_MINV: dst = e.minv; break;
    case PB_FIELD_TYPE: dst = e.type; break;
    default: return fail(h, PB_ERR_ARG, "field is read-only");
  }
  if (!dst) return fail(h, PB_ERR_STATE, "field not allocated for this handle");
  H_CUDA(cudaMemcpyAsync(dst, host, need, cudaMemcpyHostToDevice, e.stream));
  H_CUDA(cudaStreamSynchronize(e.stream));
  if (field == PB_FIELD_MINV) {
    std::vector<float> mi(e.N), m(e.N);
    std::memcpy(mi.data(), host, need);
    for (uint32_t i = 0; i < e.N; ++i) m[i] = 1.0f / mi[i];
    H_CUDA(cudaMemcpyAsync(e.mass, m.data(), need, cudaMemcpyHostToDevice, e.stream));
    H_CUDA(cudaStreamSynchronize(e.stream));
  }
  return PB_OK;
}

int pb_pool_reserve(size_t bytes) { return engine_pool_reserve(bytes); }

int pb_pool_trim(void) {
  engine_pool_trim();
  return PB_OK;
}

}  // extern "C"
