// Host implementation of the batch C ABI (include/pb/pb.h, pb_batch_*): many
// independent systems in one engine.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/pb/pb.h"
#include "engine.h"
#include "plan.h"

using namespace pb;

struct pb_batch {
  Engine e;
};

namespace {

int fail(pb_batch *b, int code, const std::string &msg) {
  if (b) b->e.err = msg;
  return code;
}

#define B_CUDA(call)                                                                   \
  do {                                                                                 \
    cudaError_t c_ = (call);                                                           \
    if (c_ != cudaSuccess)                                                             \
      return fail(b, PB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(c_)); \
  } while (0)

// Device slice of one per-atom field of system s: pointer and bytes.
int field_slice(pb_batch *b, uint32_t s, int field, char **ptr, size_t *bytes, bool for_set) {
  Engine &e = b->e;
  const size_t a0 = e.atom0[s], n = e.sp[s].n;
  switch (field) {
    case PB_FIELD_R:
      *ptr = (char *)(e.r + a0);
      *bytes = 16 * n;
      if (for_set) e.sp[s].r_set = true;
      break;
    case PB_FIELD_V:
      if (!e.v) return fail(b, PB_ERR_STATE, "batch keeps FP64 velocities");
      *ptr = (char *)(e.v + a0); *bytes = 16 * n; break;
    case PB_FIELD_VD:
      if (!e.vd) return fail(b, PB_ERR_STATE, "batch keeps FP32 velocities");
      *ptr = (char *)(e.vd + 3 * a0); *bytes = 24 * n; break;
    case PB_FIELD_F:
      *ptr = (char *)(e.F[for_set ? e.last : engine_force_buffer(e, s)] + a0);
      *bytes = 16 * n;
      break;
    case PB_FIELD_FOLD:
      // a finished system's Fold is its last force, as after any completed step
      *ptr = (char *)(e.F[engine_finished(e, s) ? engine_force_buffer(e, s) : 1 - e.cur] + a0);
      *bytes = 16 * n;
      break;
    case PB_FIELD_MINV: *ptr = (char *)(e.minv + a0); *bytes = 4 * n; break;
    case PB_FIELD_TYPE: *ptr = (char *)(e.type + a0); *bytes = 2 * n; break;
    case PB_FIELD_MASS:
      if (for_set) return fail(b, PB_ERR_ARG, "set MINV instead of MASS");
      *ptr = (char *)(e.mass + a0); *bytes = 4 * n; break;
    default: return fail(b, PB_ERR_NOTFOUND, "not a per-atom field of a batch");
  }
  return PB_OK;
}

}  // namespace

extern "C" {

int pb_batch_create(const uint32_t *natoms, uint32_t nsys, uint32_t flags, pb_batch **out) {
  if (!out || !natoms || nsys == 0) return PB_ERR_ARG;
  *out = nullptr;
  pb_batch *b = new pb_batch;
  const int rc = engine_init(b->e, natoms, nsys, flags);
  if (rc) {
    engine_free(b->e);
    delete b;
    return rc;
  }
  *out = b;
  return PB_OK;
}

int pb_batch_repack(const pb_batch *old, const int32_t *src, const uint32_t *natoms, uint32_t nsys,
                    pb_batch **out) {
  if (!old || !src || !out || nsys == 0) return PB_ERR_ARG;
  *out = nullptr;
  const Engine &o = old->e;
  std::vector<uint32_t> n(nsys);
  for (uint32_t k = 0; k < nsys; ++k) {
    if (src[k] >= 0) {
      if ((uint32_t)src[k] >= o.nsys) return PB_ERR_ARG;
      n[k] = o.sp[src[k]].n;
    } else {
      if (!natoms || natoms[k] == 0) return PB_ERR_ARG;
      n[k] = natoms[k];
    }
  }
  pb_batch *b = new pb_batch;
  Engine &e = b->e;
  int rc = engine_init(e, n.data(), nsys, o.flags, false);  // the gather below writes the state
  if (rc) {
    engine_free(e);
    delete b;
    return rc;
  }
  e.force_threads = o.force_threads;
  e.seg_scale = o.seg_scale;
  // a repack keeps the cell build its source batch measured (the particle
  // order of continuing systems does not change)
  e.cells_bucket = o.cells_bucket;
  e.cells_chosen = o.cells_chosen;
  auto bail = [&](int code) {
    engine_free(e);
    delete b;
    return code;
  };
  if (cudaStreamSynchronize(o.stream) != cudaSuccess) return bail(PB_ERR_CUDA);
  std::vector<DevScalars> osc(o.nsys), nsc(nsys);
  if (cudaMemcpy(osc.data(), o.sc, sizeof(DevScalars) * o.nsys, cudaMemcpyDeviceToHost) !=
      cudaSuccess)
    return bail(PB_ERR_CUDA);
  std::vector<uint32_t> oleft(o.nsys, 0xffffffffu), nleft(nsys, 0xffffffffu);
  if (o.steps_left && cudaMemcpy(oleft.data(), o.steps_left, 4 * (size_t)o.nsys,
                                 cudaMemcpyDeviceToHost) != cudaSuccess)
    return bail(PB_ERR_CUDA);
  e.last = o.last ^ o.cur;  // new F[k] is old F[k ^ o.cur]
  std::vector<GatherSrc> gs(nsys, GatherSrc{-1, 0, 0, 0});
  std::memset(nsc.data(), 0, sizeof(DevScalars) * nsys);
  for (uint32_t k = 0; k < nsys; ++k) {
    if (src[k] < 0) continue;
    const uint32_t s = (uint32_t)src[k];
    const size_t oa = o.atom0[s], na = e.atom0[k], cnt = n[k];
    SysParams &P = e.sp[k];
    const SysParams &Q = o.sp[s];
    std::memcpy(P.cell, Q.cell, sizeof(P.cell));
    P.cell_set = Q.cell_set;
    P.rmax = Q.rmax;
    P.rmax2 = Q.rmax2;
    P.kB = Q.kB;
    P.lj = Q.lj;
    P.lj_set = Q.lj_set;
    P.r_set = Q.r_set;  // positions are gathered from the old batch
    P.lj_percut = Q.lj_percut;
    P.m0 = Q.m0;
    P.dt = Q.dt;
    nsc[k] = osc[s];
    for (auto &c : nsc[k].counter) c = 0;
    nleft[k] = oleft[s];
    // a finished system carries its last force in both buffers (F and Fold
    // coincide after a completed step)
    const bool fin = engine_finished(o, s);
    const int fb = engine_force_buffer(o, s);
    gs[k].src = (int32_t)s;
    gs[k].o_atom0 = (uint32_t)oa;
    gs[k].fb0 = (uint8_t)(fin ? fb : o.cur);
    gs[k].fb1 = (uint8_t)(fin ? fb : 1 - o.cur);
    (void)na;
    (void)cnt;
  }
  // all continuing systems' per-atom state in one launch
  GatherSrc *d_gs = nullptr;
  if (engine_alloc_bytes(e, (void **)&d_gs, sizeof(GatherSrc) * nsys) != cudaSuccess ||
      cudaMemcpyAsync(d_gs, gs.data(), sizeof(GatherSrc) * nsys, cudaMemcpyHostToDevice,
                      e.stream) != cudaSuccess)
    return bail(PB_ERR_CUDA);
  GatherArgs ga{};
  ga.map = e.d_map;
  ga.sys = e.d_sysint;
  ga.nblocks = e.nblocks;
  ga.gs = d_gs;
  ga.o_r = o.r;
  ga.o_v = o.v;
  ga.o_F0 = o.F[0];
  ga.o_F1 = o.F[1];
  ga.o_vd = o.vd;
  ga.o_minv = o.minv;
  ga.o_mass = o.mass;
  ga.o_type = o.type;
  ga.r = e.r;
  ga.v = e.v;
  ga.F0 = e.F[0];
  ga.F1 = e.F[1];
  ga.vd = e.vd;
  ga.minv = e.minv;
  ga.mass = e.mass;
  ga.type = e.type;
  const cudaError_t gc = launch_gather_state(ga, e.stream);
  engine_free_bytes(e, d_gs);
  if (gc != cudaSuccess) return bail(PB_ERR_CUDA);
  if (cudaMemcpyAsync(e.sc, nsc.data(), sizeof(DevScalars) * nsys, cudaMemcpyHostToDevice,
                      e.stream) != cudaSuccess ||
      cudaStreamSynchronize(e.stream) != cudaSuccess)
    return bail(PB_ERR_CUDA);
  rc = engine_upload_lj(e);
  if (!rc) rc = engine_upload_sysint(e);
  if (!rc && o.steps_left) rc = engine_set_steps_left(e, nleft.data());
  if (rc) return bail(rc);
  *out = b;
  return PB_OK;
}

int pb_batch_destroy(pb_batch *b) {
  if (!b) return PB_ERR_ARG;
  engine_free(b->e);
  delete b;
  return PB_OK;
}

int pb_batch_set_stream(pb_batch *b, void *stream) {
  return b ? engine_set_stream(b->e, (cudaStream_t)stream) : PB_ERR_ARG;
}

const char *pb_batch_last_error(const pb_batch *b) { return b ? b->e.err.c_str() : "null handle"; }

int pb_batch_size(const pb_batch *b, uint32_t *nsys, uint32_t *natoms_total, uint32_t *atom0) {
  if (!b) return PB_ERR_ARG;
  if (nsys) *nsys = b->e.nsys;
  if (natoms_total) *natoms_total = b->e.N;
  if (atom0) std::memcpy(atom0, b->e.atom0.data(), 4 * (size_t)(b->e.nsys + 1));
  return PB_OK;
}

int pb_batch_set_system(pb_batch *b, uint32_t sys, const float cell6[6], float rc,
                        const float *sigma_eps, uint32_t ntypes, float dt, float kB) {
  if (!b || !cell6 || !sigma_eps || sys >= b->e.nsys) return PB_ERR_ARG;
  if (ntypes < 1 || ntypes > (uint32_t)kMaxTypes || !(rc > 0) || !(dt > 0) || !(kB > 0))
    return fail(b, PB_ERR_ARG, "bad system parameters");
  for (int k = 0; k < 3; ++k)
    if (!(cell6[2 * k + 1] > cell6[2 * k])) return fail(b, PB_ERR_ARG, "empty box");
  SysParams &P = b->e.sp[sys];
  std::memcpy(P.cell, cell6, sizeof(P.cell));
  P.cell_set = true;
  P.rmax2 = rc * rc;
  P.rmax = rc;
  lj_table_fill(P, sigma_eps, ntypes, 2, false);
  P.dt = dt;
  P.kB = kB;
  b->e.cells_ready = false;  // pb_batch_setup_cells uploads the tables of all systems
  engine_drop_graph(b->e);
  return PB_OK;
}

int pb_batch_set_lj_cut(pb_batch *b, uint32_t sys, const float *p, uint32_t ntypes) {
  if (!b || !p || sys >= b->e.nsys || ntypes < 1 || ntypes > (uint32_t)kMaxTypes)
    return PB_ERR_ARG;
  SysParams &P = b->e.sp[sys];
  if (!P.cell_set) return fail(b, PB_ERR_STATE, "pb_batch_set_system first");
  lj_table_fill(P, p, ntypes, 3, true);
  float rc2 = 0.f;
  for (uint32_t k = 0; k < ntypes * ntypes; ++k) rc2 = std::max(rc2, P.lj.rc2[k]);
  P.rmax2 = rc2;
  P.rmax = std::sqrt(rc2);
  b->e.cells_ready = false;  // uploaded by pb_batch_setup_cells
  engine_drop_graph(b->e);
  return PB_OK;
}

int pb_batch_import(pb_batch *b, uint32_t sys, const double *r3, const double *v3,
                    const double *mass, const uint32_t *type) {
  if (!b || !r3) return PB_ERR_ARG;
  return engine_import(b->e, sys, r3, v3, mass, type);
}

int pb_batch_setup_cells(pb_batch *b, const float *rmax) {
  if (!b) return PB_ERR_ARG;
  for (uint32_t s = 0; s < b->e.nsys; ++s) {
    SysParams &P = b->e.sp[s];
    if (!P.cell_set || !P.lj_set) return fail(b, PB_ERR_STATE, "pb_batch_set_system first");
    const float r = rmax ? rmax[s] : std::sqrt(P.rmax2);
    if (!(r > 0)) return fail(b, PB_ERR_ARG, "bad rmax");
    P.rmax = r;
  }
  return engine_setup_cells(b->e);
}

int pb_batch_force(pb_batch *b, uint32_t flags) {
  if (!b) return PB_ERR_ARG;
  int rc = engine_build(b->e);
  return rc ? rc : engine_force(b->e, (flags & PB_FORCE_ENERGY) != 0);
}

int pb_batch_clear_force(pb_batch *b) { return b ? engine_clear_force(b->e) : PB_ERR_ARG; }

int pb_batch_run(pb_batch *b, int mode, uint32_t steps) {
  return b ? engine_run(b->e, mode, steps) : PB_ERR_ARG;
}

int pb_batch_run_timed(pb_batch *b, int mode, uint32_t steps, float *ms) {
  if (!b || !ms) return PB_ERR_ARG;
  cudaEvent_t x, y;
  B_CUDA(cudaEventCreate(&x));
  B_CUDA(cudaEventCreate(&y));
  B_CUDA(cudaEventRecord(x, b->e.stream));
  const int rc = engine_run(b->e, mode, steps);
  cudaEventRecord(y, b->e.stream);
  cudaEventSynchronize(y);
  cudaEventElapsedTime(ms, x, y);
  cudaEventDestroy(x);
  cudaEventDestroy(y);
  return rc;
}

int pb_batch_profile(pb_batch *b, int mode, uint32_t steps, double ms[3]) {
  if (!b || !ms || steps == 0) return PB_ERR_ARG;
  return engine_profile(b->e, mode, steps, ms);
}

int pb_batch_set_steps_left(pb_batch *b, const uint32_t *steps) {
  return b ? engine_set_steps_left(b->e, steps) : PB_ERR_ARG;
}

int pb_batch_get_steps_left(pb_batch *b, uint32_t *steps) {
  return (b && steps) ? engine_get_steps_left(b->e, steps) : PB_ERR_ARG;
}

int pb_batch_reduce(pb_batch *b, pb_md_sums *out) {
  if (!b || !out) return PB_ERR_ARG;
  int rc = engine_mv2(b->e);
  if (!rc) rc = engine_fv(b->e);
  std::vector<DevScalars> sc;
  if (!rc) rc = engine_scalars(b->e, sc);
  if (rc) return rc;
  for (uint32_t s = 0; s < b->e.nsys; ++s) {
    out[s].mv2 = sc[s].mv2;
    out[s].fv = sc[s].fv;
    out[s].pe = b->e.energy_valid ? sc[s].pe : NAN;
    out[s].pe_shift = b->e.energy_valid ? sc[s].pe_shift : NAN;
    out[s].virial = b->e.energy_valid ? sc[s].virial : NAN;
    out[s].xi = sc[s].xi_old;
  }
  return PB_OK;
}

int pb_batch_temperature(pb_batch *b, double *T) {
  if (!b || !T) return PB_ERR_ARG;
  int rc = engine_mv2(b->e);
  std::vector<DevScalars> sc;
  if (!rc) rc = engine_scalars(b->e, sc);
  if (rc) return rc;
  for (uint32_t s = 0; s < b->e.nsys; ++s)
    T[s] = sc[s].mv2 / (3.0 * b->e.sp[s].n * b->e.sp[s].kB);
  return PB_OK;
}

int pb_batch_status(pb_batch *b, uint32_t *bits) {
  if (!b || !bits) return PB_ERR_ARG;
  std::vector<uint32_t> v;
  const int rc = engine_status(b->e, v);
  if (rc) return rc;
  std::memcpy(bits, v.data(), 4 * v.size());
  return PB_OK;
}

int pb_batch_scale_velocities(pb_batch *b, const double *s) {
  return (b && s) ? engine_scale(b->e, s) : PB_ERR_ARG;
}

int pb_batch_adjust_velocities(pb_batch *b, const double *v1) {
  return (b && v1) ? engine_adjust(b->e, v1) : PB_ERR_ARG;
}

int pb_batch_get(pb_batch *b, uint32_t sys, int field, void *host, size_t bytes) {
  if (!b || !host || sys >= b->e.nsys) return PB_ERR_ARG;
  char *p = nullptr;
  size_t need = 0;
  const int rc = field_slice(b, sys, field, &p, &need, false);
  if (rc) return rc;
  if (bytes != need) return fail(b, PB_ERR_ARG, "size mismatch for field");
  B_CUDA(cudaMemcpyAsync(host, p, need, cudaMemcpyDeviceToHost, b->e.stream));
  B_CUDA(cudaStreamSynchronize(b->e.stream));
  return PB_OK;
}

int pb_batch_set(pb_batch *b, uint32_t sys, int field, const void *host, size_t bytes) {
  if (!b || !host || sys >= b->e.nsys) return PB_ERR_ARG;
  char *p = nullptr;
  size_t need = 0;
  const int rc = field_slice(b, sys, field, &p, &need, true);
  if (rc) return rc;
  if (bytes != need) return fail(b, PB_ERR_ARG, "size mismatch for field");
  B_CUDA(cudaMemcpyAsync(p, host, need, cudaMemcpyHostToDevice, b->e.stream));
  if (field == PB_FIELD_MINV) {
    const uint32_t n = b->e.sp[sys].n;
    std::vector<float> mi(n), m(n);
    std::memcpy(mi.data(), host, need);
    for (uint32_t i = 0; i < n; ++i) m[i] = 1.0f / mi[i];
    B_CUDA(cudaMemcpyAsync(b->e.mass + b->e.atom0[sys], m.data(), need, cudaMemcpyHostToDevice,
                           b->e.stream));
  }
  B_CUDA(cudaStreamSynchronize(b->e.stream));
  return PB_OK;
}

int pb_batch_set_tuning(pb_batch *b, int force_threads, float seg_scale) {
  if (!b) return PB_ERR_ARG;
  if (force_threads != 128 && force_threads != 256) return fail(b, PB_ERR_ARG, "threads 128|256");
  if (!(seg_scale > 0.05f && seg_scale < 20.f)) return fail(b, PB_ERR_ARG, "bad seg_scale");
  b->e.force_threads = force_threads;
  b->e.seg_scale = seg_scale;
  b->e.cells_ready = false;
  engine_drop_graph(b->e);
  return PB_OK;
}

int pb_batch_estimate_bytes(const uint32_t *natoms, const float *cells6, const float *rmax,
                            uint32_t nsys, uint32_t flags, size_t *bytes) {
  if (!natoms || !cells6 || !rmax || !bytes || nsys == 0) return PB_ERR_ARG;
  // per atom: r, F[2], rs (16 B each), minv, mass, key, pid_tmp, pid, slot
  // (4 B each), the overflow list entry (8 B), x, y, z, type mirrors of rs
  // (16 B), type (2 B), velocities (16 or 24 B), sysid (4 B), and for the
  // half-shell kernel its fixed-point force sums (48 B)
  const bool half = (flags & PB_MD_HALF_SHELL) && !(flags & PB_MD_ACC_FP64);
  const size_t per_atom = 16 * 4 + 4 * 6 + 8 + 16 + 2 + ((flags & PB_MD_VEL_FP64) ? 24 : 16) +
                          (nsys > 1 ? 4 : 0) + (half ? 48 : 0);
  // per cell: the bucket, sized by the densest system as the engine does
  double apc_max = 0.0;
  for (uint32_t s = 0; s < nsys; ++s) {
    Grid g;
    if (!make_grid(cells6 + 6 * s, rmax[s], g)) return PB_ERR_ARG;
    apc_max = std::max(apc_max, (double)natoms[s] / g.ncells);
  }
  const size_t per_cell_bucket = 4 * (size_t)choose_bucket_cap(apc_max) + 1;  // + tile count
  size_t total = 0;
  for (uint32_t s = 0; s < nsys; ++s) {
    Grid g;
    if (!make_grid(cells6 + 6 * s, rmax[s], g)) return PB_ERR_ARG;
    total += per_cell_bucket * (size_t)g.ncells;
    const size_t cols = (size_t)g.n[0] * g.n[1];
    const size_t items = cols * (size_t)(2 + g.n[2] / 4);  // generous: runs per column
    const size_t blocks = blocks_for(natoms[s]);
    total += per_atom * natoms[s] + 64 + 8 * (size_t)g.ncells + 8 * cols +
             (sizeof(ForceItem) + 32) * items + (sizeof(BlockMap) + 64) * blocks +
             sizeof(SysDesc) + sizeof(SysInt) + sizeof(DevScalars) + sizeof(LJTable) + 64;
  }
  *bytes = total + (1u << 20);  // allocation granularity and small tables
  return PB_OK;
}

}  // extern "C"
