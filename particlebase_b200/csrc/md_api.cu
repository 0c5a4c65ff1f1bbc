// Host implementation of the single-system C ABI (include/pb/pb.h).
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/pb/pb.h"
#include "integrate.cuh"
#include "md.cuh"
#include "plan.h"

using namespace pb;

static_assert(sizeof(pb_particle) == 96, "pb_particle must match ParticleBase");
static_assert(offsetof(pb_particle, is_fixed) == 56, "pb_particle layout");
static_assert(offsetof(pb_particle, a) == 64, "pb_particle layout");
static_assert(offsetof(pb_particle, type) == 88, "pb_particle layout");

struct pb_md {
  uint32_t N = 0;
  uint32_t flags = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::string err;

  float cell[6] = {0, 1, 0, 1, 0, 1};
  bool cell_set = false;
  float rmax = 0.f, rmax2 = 0.f;
  float kB = 1.f;
  LJTable lj{};
  bool lj_set = false, lj_percut = false;
  Grid grid{};
  bool cells_ready = false;
  double m0 = 1.0;
  int seg = 1, cap = 0;
  int force_threads = 256;
  std::vector<uint32_t> key_of_ref;   // reference cell id -> key
  std::vector<uint32_t> ref_of_key;   // key -> reference cell id

  // device state
  float4 *r = nullptr, *v = nullptr, *F[2] = {nullptr, nullptr}, *rs = nullptr;
  int cur = 0;  // F[cur] is F(t), F[1 - cur] is Fold
  double *vd = nullptr;
  float *minv = nullptr, *mass = nullptr;
  uint16_t *type = nullptr;
  uint32_t *key = nullptr, *within = nullptr, *count = nullptr, *start = nullptr,
           *tilesum = nullptr, *pid_tmp = nullptr, *pid = nullptr, *slot = nullptr;
  uint32_t *colrank = nullptr, *colxy = nullptr;
  SysDesc *d_sys = nullptr;
  LJTable *d_lj = nullptr;
  ForceItem *d_items = nullptr;
  uint32_t nitems = 0;
  double *fpartials = nullptr;   // force energy partials, 4 per item
  double *ipartials = nullptr;   // integrator partials, 8 per block
  DevScalars *sc = nullptr;
  uint32_t *status = nullptr;
  bool energy_valid = false;

  // CUDA graph of two whole steps (F ping-pong returns to the same parity)
  cudaGraphExec_t graph = nullptr;
  float graph_dt = 0.f;
  int graph_mode = -1;
};

namespace {

int fail(pb_md *h, int code, const std::string &msg) {
  if (h) h->err = msg;
  return code;
}

int cuda_fail(pb_md *h, cudaError_t e, const char *what) {
  return fail(h, PB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define PB_CUDA(call)                                   \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) return cuda_fail(h, e_, #call); \
  } while (0)

template <typename T>
cudaError_t dalloc(T **p, size_t count) {
  if (count == 0) count = 1;
  return cudaMalloc((void **)p, sizeof(T) * count);
}

template <typename T>
void dfree(T *&p) {
  if (p) cudaFree((void *)p);
  p = nullptr;
}

void free_cells(pb_md *h) {
  dfree(h->key);
  dfree(h->within);
  dfree(h->count);
  dfree(h->start);
  dfree(h->tilesum);
  dfree(h->pid_tmp);
  dfree(h->pid);
  dfree(h->slot);
  dfree(h->rs);
  dfree(h->colrank);
  dfree(h->colxy);
  dfree(h->d_sys);
  dfree(h->d_items);
  dfree(h->fpartials);
  h->cells_ready = false;
}

void drop_graph(pb_md *h) {
  if (h->graph) cudaGraphExecDestroy(h->graph);
  h->graph = nullptr;
  h->graph_mode = -1;
}

IntegrateArgs iargs(pb_md *h, float dt, int wrap) {
  IntegrateArgs a{};
  a.r = h->r;
  a.v = h->vd ? nullptr : h->v;
  a.vd = h->vd;
  a.F = h->F[h->cur];
  a.Fold = h->F[1 - h->cur];
  a.minv = h->minv;
  a.mass = h->mass;
  a.N = h->N;
  a.dt = dt;
  for (int k = 0; k < 3; ++k) {
    a.c0[k] = h->cell[2 * k];
    a.c1[k] = h->cell[2 * k + 1];
    a.L[k] = h->cell[2 * k + 1] - h->cell[2 * k];
  }
  a.wrap = wrap;
  a.sc = h->sc;
  a.partials = h->ipartials;
  a.status = h->status;
  return a;
}

CellBufs cbufs(pb_md *h) {
  CellBufs b{};
  b.r = h->r;
  b.type = h->type;
  b.sysid = nullptr;
  b.sys = h->d_sys;
  b.colrank = h->colrank;
  b.N = h->N;
  b.ncells = h->grid.ncells;
  b.key = h->key;
  b.within = h->within;
  b.count = h->count;
  b.start = h->start;
  b.tilesum = h->tilesum;
  b.pid_tmp = h->pid_tmp;
  b.pid = h->pid;
  b.slot = h->slot;
  b.rs = h->rs;
  b.status = h->status;
  return b;
}

ForceBufs fbufs(pb_md *h) {
  ForceBufs b{};
  b.rs = h->rs;
  b.start = h->start;
  b.pid = h->pid;
  b.sys = h->d_sys;
  b.colxy = h->colxy;
  b.colrank = h->colrank;
  b.lj = h->d_lj;
  b.items = h->d_items;
  b.nitems = h->nitems;
  b.cap = h->cap;
  b.F = h->F[h->cur];
  b.partials = h->fpartials;
  b.status = h->status;
  return b;
}

bool ready(pb_md *h) { return h && h->cells_ready && h->lj_set && h->N > 0; }

int do_build(pb_md *h) {
  cudaError_t e = launch_cell_build(cbufs(h), h->stream);
  if (e != cudaSuccess) return cuda_fail(h, e, "cell build");
  return PB_OK;
}

int do_force(pb_md *h, bool energy) {
  cudaError_t e = launch_force(fbufs(h), h->lj.nt, energy, (h->flags & PB_MD_ACC_FP64) != 0,
                               h->force_threads, h->stream);
  if (e != cudaSuccess) return cuda_fail(h, e, "force");
  if (energy) {
    e = launch_energy_total(h->fpartials, h->nitems, h->sc, h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "energy total");
  }
  h->energy_valid = energy;
  return PB_OK;
}

int do_evolve(pb_md *h, float dt, int mode, int wrap) {
  IntegrateArgs a = iargs(h, dt, wrap);
  cudaError_t e;
  if (mode == PB_MODE_VV) {
    if (h->vd) return fail(h, PB_ERR_UNSUPPORTED, "velocity Verlet uses FP32 velocities");
    e = launch_vv(a, h->stream);
  } else {
    e = launch_gauss(a, h->stream);
  }
  if (e != cudaSuccess) return cuda_fail(h, e, "time evolution");
  h->cur = 1 - h->cur;
  return PB_OK;
}

int do_step(pb_md *h, float dt, int mode) {
  int rc = do_build(h);
  if (rc) return rc;
  rc = do_force(h, false);
  if (rc) return rc;
  return do_evolve(h, dt, mode, 1);
}

}  // namespace

extern "C" {

const char *pb_version(void) { return "particlebase_b200 0.1 (sm_100a)"; }

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
  h->N = n;
  h->flags = flags;
  cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete h;
    return PB_ERR_CUDA;
  }
  h->own_stream = true;
  bool ok = dalloc(&h->r, n) == cudaSuccess && dalloc(&h->F[0], n) == cudaSuccess &&
            dalloc(&h->F[1], n) == cudaSuccess && dalloc(&h->minv, n) == cudaSuccess &&
            dalloc(&h->mass, n) == cudaSuccess && dalloc(&h->type, n) == cudaSuccess &&
            dalloc(&h->sc, 1) == cudaSuccess && dalloc(&h->status, 1) == cudaSuccess &&
            dalloc(&h->d_lj, 1) == cudaSuccess &&
            dalloc(&h->ipartials, (size_t)8 * integrate_blocks(n)) == cudaSuccess;
  if (flags & PB_MD_VEL_FP64)
    ok = ok && dalloc(&h->vd, (size_t)3 * n) == cudaSuccess;
  else
    ok = ok && dalloc(&h->v, n) == cudaSuccess;
  if (!ok) {
    pb_md_destroy(h);
    return PB_ERR_OOM;
  }
  cudaMemsetAsync(h->r, 0, sizeof(float4) * n, h->stream);
  cudaMemsetAsync(h->F[0], 0, sizeof(float4) * n, h->stream);
  cudaMemsetAsync(h->F[1], 0, sizeof(float4) * n, h->stream);
  if (h->v) cudaMemsetAsync(h->v, 0, sizeof(float4) * n, h->stream);
  if (h->vd) cudaMemsetAsync(h->vd, 0, sizeof(double) * 3 * n, h->stream);
  cudaMemsetAsync(h->type, 0, sizeof(uint16_t) * n, h->stream);
  cudaMemsetAsync(h->sc, 0, sizeof(DevScalars), h->stream);
  cudaMemsetAsync(h->status, 0, sizeof(uint32_t), h->stream);
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) {
    pb_md_destroy(h);
    return PB_ERR_CUDA;
  }
  *out = h;
  return PB_OK;
}

int pb_md_destroy(pb_md *h) {
  if (!h) return PB_ERR_ARG;
  if (h->stream) cudaStreamSynchronize(h->stream);
  drop_graph(h);
  free_cells(h);
  dfree(h->r);
  dfree(h->v);
  dfree(h->vd);
  dfree(h->F[0]);
  dfree(h->F[1]);
  dfree(h->minv);
  dfree(h->mass);
  dfree(h->type);
  dfree(h->sc);
  dfree(h->status);
  dfree(h->d_lj);
  dfree(h->ipartials);
  if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return PB_OK;
}

int pb_md_set_stream(pb_md *h, void *stream) {
  if (!h) return PB_ERR_ARG;
  PB_CUDA(cudaStreamSynchronize(h->stream));
  drop_graph(h);
  if (h->own_stream) cudaStreamDestroy(h->stream);
  h->stream = (cudaStream_t)stream;
  h->own_stream = false;
  return PB_OK;
}

const char *pb_md_last_error(const pb_md *h) { return h ? h->err.c_str() : "null handle"; }

int pb_md_status(pb_md *h, uint32_t *bits) {
  if (!h || !bits) return PB_ERR_ARG;
  PB_CUDA(cudaMemcpyAsync(bits, h->status, sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
  PB_CUDA(cudaStreamSynchronize(h->stream));
  PB_CUDA(cudaMemsetAsync(h->status, 0, sizeof(uint32_t), h->stream));
  return PB_OK;
}

int pb_md_set_cell(pb_md *h, const float cell6[6]) {
  if (!h || !cell6) return PB_ERR_ARG;
  for (int k = 0; k < 3; ++k)
    if (!(cell6[2 * k + 1] > cell6[2 * k])) return fail(h, PB_ERR_ARG, "empty box");
  std::memcpy(h->cell, cell6, sizeof(float) * 6);
  h->cell_set = true;
  if (h->cells_ready) free_cells(h);  // the grid depends on the box
  drop_graph(h);
  return PB_OK;
}

static int upload_lj(pb_md *h) {
  PB_CUDA(cudaMemcpyAsync(h->d_lj, &h->lj, sizeof(LJTable), cudaMemcpyHostToDevice, h->stream));
  PB_CUDA(cudaStreamSynchronize(h->stream));
  drop_graph(h);
  return PB_OK;
}

static void fill_lj(pb_md *h, const float *p, uint32_t nt, int stride, bool percut) {
  LJTable &t = h->lj;
  std::memset(&t, 0, sizeof(t));
  t.nt = (int)nt;
  for (uint32_t a = 0; a < nt; ++a)
    for (uint32_t b = 0; b < nt; ++b) {
      const uint32_t k = a * nt + b;
      const float sig = p[stride * k], eps = p[stride * k + 1];
      t.s2[k] = sig * sig;         // _setLJparams: sigma^2
      t.e24[k] = eps * 24.0f;      // _setLJparams: 24 epsilon
      t.e4[k] = eps * 4.0f;
      const float rc2 = percut ? p[stride * k + 2] * p[stride * k + 2] : h->rmax2;
      t.rc2[k] = rc2;
      const double sr6 = rc2 > 0 ? std::pow((double)t.s2[k] / rc2, 3) : 0.0;
      t.ushift[k] = (float)(4.0 * eps * (sr6 * sr6 - sr6));
    }
}

int pb_md_set_lj(pb_md *h, const float *sigma_eps, uint32_t ntypes) {
  if (!h || !sigma_eps || ntypes < 1 || ntypes > (uint32_t)kMaxTypes) return PB_ERR_ARG;
  fill_lj(h, sigma_eps, ntypes, 2, false);
  h->lj_set = true;
  h->lj_percut = false;
  return upload_lj(h);
}

int pb_md_set_lj_cut(pb_md *h, const float *p, uint32_t ntypes) {
  if (!h || !p || ntypes < 1 || ntypes > (uint32_t)kMaxTypes) return PB_ERR_ARG;
  fill_lj(h, p, ntypes, 3, true);
  h->lj_set = true;
  h->lj_percut = true;
  return upload_lj(h);
}

int pb_md_set_rmax2(pb_md *h, float rmax2) {
  if (!h || !(rmax2 > 0)) return PB_ERR_ARG;
  h->rmax2 = rmax2;
  if (h->lj_set && !h->lj_percut) {
    for (int k = 0; k < h->lj.nt * h->lj.nt; ++k) {
      h->lj.rc2[k] = rmax2;
      const double sr6 = std::pow((double)h->lj.s2[k] / rmax2, 3);
      h->lj.ushift[k] = (float)((double)h->lj.e4[k] * (sr6 * sr6 - sr6));
    }
    return upload_lj(h);
  }
  return PB_OK;
}

int pb_md_set_kB(pb_md *h, float kB) {
  if (!h || !(kB > 0)) return PB_ERR_ARG;
  h->kB = kB;
  return PB_OK;
}

int pb_md_import_arrays(pb_md *h, const double *r3, const double *v3, const double *mass,
                        const uint32_t *type) {
  if (!h || !r3) return PB_ERR_ARG;
  const uint32_t N = h->N;
  std::vector<float4> r4(N), v4(N, make_float4(0, 0, 0, 0));
  std::vector<float> minv(N, 1.f), m(N, 1.f);
  std::vector<uint16_t> t(N, 0);
  std::vector<double> vd;
  double msum = 0;
  for (uint32_t i = 0; i < N; ++i) {
    r4[i] = make_float4((float)r3[3 * i], (float)r3[3 * i + 1], (float)r3[3 * i + 2], 0.f);
    if (v3) v4[i] = make_float4((float)v3[3 * i], (float)v3[3 * i + 1], (float)v3[3 * i + 2], 0.f);
    const double mi = mass ? mass[i] : 1.0;
    if (!(mi > 0)) return fail(h, PB_ERR_ARG, "mass must be positive");
    minv[i] = (float)(1.0 / mi);       // cudaParticleBase::import: TMP[i] = 1.0 / m
    m[i] = 1.0f / minv[i];             // cudaParticleMD::setM: m = 1 / minv
    msum += mi;
    if (type) {
      if (type[i] >= (uint32_t)kMaxTypes) return fail(h, PB_ERR_ARG, "type id >= 8");
      t[i] = (uint16_t)type[i];
    }
  }
  h->m0 = msum / N;
  PB_CUDA(cudaMemcpyAsync(h->r, r4.data(), sizeof(float4) * N, cudaMemcpyHostToDevice, h->stream));
  PB_CUDA(cudaMemcpyAsync(h->minv, minv.data(), sizeof(float) * N, cudaMemcpyHostToDevice, h->stream));
  PB_CUDA(cudaMemcpyAsync(h->mass, m.data(), sizeof(float) * N, cudaMemcpyHostToDevice, h->stream));
  PB_CUDA(cudaMemcpyAsync(h->type, t.data(), sizeof(uint16_t) * N, cudaMemcpyHostToDevice, h->stream));
  if (h->vd) {
    vd.assign((size_t)3 * N, 0.0);
    if (v3)
      for (uint32_t i = 0; i < N; ++i)
        for (int k = 0; k < 3; ++k) vd[(size_t)k * N + i] = v3[3 * i + k];
    PB_CUDA(cudaMemcpyAsync(h->vd, vd.data(), sizeof(double) * 3 * N, cudaMemcpyHostToDevice, h->stream));
  } else {
    PB_CUDA(cudaMemcpyAsync(h->v, v4.data(), sizeof(float4) * N, cudaMemcpyHostToDevice, h->stream));
  }
  PB_CUDA(cudaStreamSynchronize(h->stream));
  return PB_OK;
}

int pb_md_import(pb_md *h, const pb_particle *p, uint32_t n) {
  if (!h || !p || n != h->N) return PB_ERR_ARG;
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
  if (!periodic) return fail(h, PB_ERR_UNSUPPORTED, "only periodic boxes are supported");
  if (!h->cell_set) return fail(h, PB_ERR_STATE, "set the cell first");
  Grid g;
  if (!make_grid(h->cell, rmax, g))
    return fail(h, PB_ERR_ARG, "cell grid needs at least 3 cells per axis (blocknum > 2)");
  free_cells(h);
  drop_graph(h);
  h->grid = g;
  h->rmax = rmax;
  const uint32_t N = h->N, C = g.ncells;
  const double apc = (double)N / C;
  h->seg = choose_segment(apc, g.n[2]);
  if (const char *e = std::getenv("PB_FORCE_THREADS")) h->force_threads = std::atoi(e);
  h->cap = choose_capacity(apc, h->seg);
  std::vector<uint32_t> rank, xy;
  morton_columns(g.n[0], g.n[1], rank, xy);
  std::vector<ForceItem> items;
  append_items(0, g, h->seg, 0, rank, xy, items);
  h->nitems = (uint32_t)items.size();
  // key <-> reference cell id maps
  h->key_of_ref.assign(C, 0);
  h->ref_of_key.assign(C, 0);
  for (int d0 = 0; d0 < g.n[0]; ++d0)
    for (int d1 = 0; d1 < g.n[1]; ++d1)
      for (int d2 = 0; d2 < g.n[2]; ++d2) {
        const uint32_t ref = d2 + d1 * g.n[2] + d0 * g.n[2] * g.n[1];
        const uint32_t key = rank[d0 * g.n[1] + d1] * g.n[2] + d2;
        h->key_of_ref[ref] = key;
        h->ref_of_key[key] = ref;
      }
  SysDesc sd{};
  sd.g = g;
  sd.atom0 = 0;
  sd.natoms = N;
  sd.cell0 = 0;
  sd.col0 = 0;
  sd.vd0 = 0;
  sd.lj = 0;
  const uint32_t ntiles = (C + 4095) / 4096;
  bool ok = dalloc(&h->key, N) == cudaSuccess && dalloc(&h->within, N) == cudaSuccess &&
            dalloc(&h->count, C) == cudaSuccess && dalloc(&h->start, (size_t)C + 1) == cudaSuccess &&
            dalloc(&h->tilesum, ntiles) == cudaSuccess && dalloc(&h->pid_tmp, N) == cudaSuccess &&
            dalloc(&h->pid, N) == cudaSuccess && dalloc(&h->slot, N) == cudaSuccess &&
            dalloc(&h->rs, N) == cudaSuccess && dalloc(&h->colrank, rank.size()) == cudaSuccess &&
            dalloc(&h->colxy, xy.size()) == cudaSuccess && dalloc(&h->d_sys, 1) == cudaSuccess &&
            dalloc(&h->d_items, items.size()) == cudaSuccess &&
            dalloc(&h->fpartials, (size_t)4 * items.size()) == cudaSuccess;
  if (!ok) {
    free_cells(h);
    return fail(h, PB_ERR_OOM, "cell list allocation failed");
  }
  PB_CUDA(cudaMemsetAsync(h->count, 0, sizeof(uint32_t) * C, h->stream));
  PB_CUDA(cudaMemcpyAsync(h->colrank, rank.data(), 4 * rank.size(), cudaMemcpyHostToDevice, h->stream));
  PB_CUDA(cudaMemcpyAsync(h->colxy, xy.data(), 4 * xy.size(), cudaMemcpyHostToDevice, h->stream));
  PB_CUDA(cudaMemcpyAsync(h->d_sys, &sd, sizeof(SysDesc), cudaMemcpyHostToDevice, h->stream));
  PB_CUDA(cudaMemcpyAsync(h->d_items, items.data(), sizeof(ForceItem) * items.size(),
                          cudaMemcpyHostToDevice, h->stream));
  PB_CUDA(cudaStreamSynchronize(h->stream));
  h->cells_ready = true;
  return PB_OK;
}

int pb_md_grid(const pb_md *h, uint32_t n3[3], float len3[3], uint32_t *ncells) {
  if (!h || !h->cells_ready) return PB_ERR_STATE;
  for (int k = 0; k < 3; ++k) {
    if (n3) n3[k] = (uint32_t)h->grid.n[k];
    if (len3) len3[k] = h->grid.len[k];
  }
  if (ncells) *ncells = h->grid.ncells;
  return PB_OK;
}

int pb_md_build_cells(pb_md *h) {
  if (!h) return PB_ERR_ARG;
  if (!h->cells_ready) return fail(h, PB_ERR_STATE, "setup_cells first");
  return do_build(h);
}

int pb_md_force(pb_md *h, uint32_t flags) {
  if (!ready(h)) return fail(h, PB_ERR_STATE, "need cell, LJ parameters and setup_cells");
  return do_force(h, (flags & PB_FORCE_ENERGY) != 0);
}

int pb_md_clear_force(pb_md *h) {
  if (!h) return PB_ERR_ARG;
  PB_CUDA(cudaMemsetAsync(h->F[0], 0, sizeof(float4) * h->N, h->stream));
  PB_CUDA(cudaMemsetAsync(h->F[1], 0, sizeof(float4) * h->N, h->stream));
  return PB_OK;
}

int pb_md_step_vv(pb_md *h, float dt) {
  if (!h) return PB_ERR_ARG;
  return do_evolve(h, dt, PB_MODE_VV, 0);
}

int pb_md_step_gauss(pb_md *h, float dt, double tol) {
  (void)tol;
  if (!h) return PB_ERR_ARG;
  return do_evolve(h, dt, PB_MODE_GAUSS, 0);
}

int pb_md_wrap(pb_md *h) {
  if (!h) return PB_ERR_ARG;
  cudaError_t e = launch_wrap(iargs(h, 0.f, 1), h->stream);
  if (e != cudaSuccess) return cuda_fail(h, e, "wrap");
  return PB_OK;
}

int pb_md_run(pb_md *h, float dt, int mode, uint32_t steps) {
  if (!ready(h)) return fail(h, PB_ERR_STATE, "need cell, LJ parameters and setup_cells");
  if (mode != PB_MODE_VV && mode != PB_MODE_GAUSS) return PB_ERR_ARG;
  if (mode == PB_MODE_VV && h->vd) return fail(h, PB_ERR_UNSUPPORTED, "VV needs FP32 velocities");
  uint32_t done = 0;
  if (steps >= 2) {
    if (!h->graph || h->graph_dt != dt || h->graph_mode != mode) {
      drop_graph(h);
      cudaGraph_t g = nullptr;
      const int cur0 = h->cur;
      PB_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
      int rc = do_step(h, dt, mode);
      if (!rc) rc = do_step(h, dt, mode);
      cudaError_t e = cudaStreamEndCapture(h->stream, &g);
      h->cur = cur0;
      if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
      }
      if (e != cudaSuccess) return cuda_fail(h, e, "graph capture");
      e = cudaGraphInstantiate(&h->graph, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) {
        h->graph = nullptr;
        return cuda_fail(h, e, "graph instantiate");
      }
      h->graph_dt = dt;
      h->graph_mode = mode;
    }
    for (; done + 2 <= steps; done += 2) PB_CUDA(cudaGraphLaunch(h->graph, h->stream));
  }
  for (; done < steps; ++done) {
    int rc = do_step(h, dt, mode);
    if (rc) return rc;
  }
  h->energy_valid = false;
  return PB_OK;
}

int pb_md_run_timed(pb_md *h, float dt, int mode, uint32_t steps, float *ms) {
  if (!h || !ms) return PB_ERR_ARG;
  cudaEvent_t a, b;
  PB_CUDA(cudaEventCreate(&a));
  PB_CUDA(cudaEventCreate(&b));
  PB_CUDA(cudaEventRecord(a, h->stream));
  int rc = pb_md_run(h, dt, mode, steps);
  cudaEventRecord(b, h->stream);
  cudaEventSynchronize(b);
  cudaEventElapsedTime(ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return rc;
}

int pb_md_profile(pb_md *h, float dt, int mode, uint32_t steps, double ms[3]) {
  if (!ready(h) || !ms || steps == 0) return PB_ERR_ARG;
  cudaEvent_t ev[4];
  for (auto &e : ev) PB_CUDA(cudaEventCreate(&e));
  double acc[3] = {0, 0, 0};
  int rc = PB_OK;
  for (uint32_t k = 0; k < steps && !rc; ++k) {
    cudaEventRecord(ev[0], h->stream);
    rc = do_build(h);
    cudaEventRecord(ev[1], h->stream);
    if (!rc) rc = do_force(h, false);
    cudaEventRecord(ev[2], h->stream);
    if (!rc) rc = do_evolve(h, dt, mode, 1);
    cudaEventRecord(ev[3], h->stream);
    cudaEventSynchronize(ev[3]);
    for (int p = 0; p < 3; ++p) {
      float t = 0;
      cudaEventElapsedTime(&t, ev[p], ev[p + 1]);
      acc[p] += t;
    }
  }
  for (auto &e : ev) cudaEventDestroy(e);
  for (int p = 0; p < 3; ++p) ms[p] = acc[p] / steps;
  return rc;
}

int pb_md_pair_stats(pb_md *h, double out[2]) {
  if (!h || !out || !h->cells_ready) return PB_ERR_STATE;
  const uint32_t C = h->grid.ncells;
  std::vector<uint32_t> start(C + 1);
  PB_CUDA(cudaMemcpyAsync(start.data(), h->start, 4 * (size_t)(C + 1), cudaMemcpyDeviceToHost,
                          h->stream));
  double np = 0;
  PB_CUDA(cudaMemcpyAsync(&np, &h->sc->npairs, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  PB_CUDA(cudaStreamSynchronize(h->stream));
  std::vector<uint32_t> nb;
  neighbor_table(h->grid, nb);
  double cand = 0;
  for (uint32_t ref = 0; ref < C; ++ref) {
    const uint32_t k = h->key_of_ref[ref];
    const double nc = start[k + 1] - start[k];
    double around = 0;
    for (int j = 0; j < 27; ++j) {
      const uint32_t kn = h->key_of_ref[nb[(size_t)ref * 27 + j]];
      around += start[kn + 1] - start[kn];
    }
    cand += nc * (around - 1.0);
  }
  out[0] = cand;
  out[1] = h->energy_valid ? np : NAN;
  return PB_OK;
}

int pb_md_reduce(pb_md *h, pb_md_sums *out) {
  if (!h || !out) return PB_ERR_ARG;
  IntegrateArgs a = iargs(h, 0.f, 0);
  cudaError_t e = launch_mv2(a, h->stream);
  if (e == cudaSuccess) e = launch_fv(a, h->stream);
  if (e != cudaSuccess) return cuda_fail(h, e, "reduce");
  DevScalars sc;
  PB_CUDA(cudaMemcpyAsync(&sc, h->sc, sizeof(sc), cudaMemcpyDeviceToHost, h->stream));
  PB_CUDA(cudaStreamSynchronize(h->stream));
  out->mv2 = sc.mv2;
  out->fv = sc.fv;
  out->pe = h->energy_valid ? sc.pe : NAN;
  out->pe_shift = h->energy_valid ? sc.pe_shift : NAN;
  out->virial = h->energy_valid ? sc.virial : NAN;
  out->xi = sc.xi_old;
  return PB_OK;
}

int pb_md_temperature(pb_md *h, double *T) {
  if (!h || !T) return PB_ERR_ARG;
  cudaError_t e = launch_mv2(iargs(h, 0.f, 0), h->stream);
  if (e != cudaSuccess) return cuda_fail(h, e, "mv2");
  double mv2 = 0;
  PB_CUDA(cudaMemcpyAsync(&mv2, &h->sc->mv2, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  PB_CUDA(cudaStreamSynchronize(h->stream));
  *T = mv2 / (3.0 * h->N * h->kB);
  return PB_OK;
}

int pb_md_scale_velocities(pb_md *h, double s) {
  if (!h) return PB_ERR_ARG;
  cudaError_t e = launch_scale(iargs(h, 0.f, 0), s, h->stream);
  if (e != cudaSuccess) return cuda_fail(h, e, "scale");
  return PB_OK;
}

int pb_md_adjust_velocities(pb_md *h, double v1) {
  if (!h) return PB_ERR_ARG;
  cudaError_t e = launch_adjust(iargs(h, 0.f, 0), v1, h->stream);
  if (e != cudaSuccess) return cuda_fail(h, e, "adjust");
  return PB_OK;
}

int pb_md_mean_mass(const pb_md *h, double *m0) {
  if (!h || !m0) return PB_ERR_ARG;
  *m0 = h->m0;
  return PB_OK;
}

int pb_md_size(const pb_md *h, uint32_t *n) {
  if (!h || !n) return PB_ERR_ARG;
  *n = h->N;
  return PB_OK;
}

int pb_md_field_bytes(const pb_md *h, int field, size_t *bytes) {
  if (!h || !bytes) return PB_ERR_ARG;
  const size_t N = h->N, C = h->grid.ncells;
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
  size_t need = 0;
  int rc = pb_md_field_bytes(h, field, &need);
  if (rc) return rc;
  if (bytes != need) return fail(h, PB_ERR_ARG, "size mismatch for field");
  const bool cell_field = field >= PB_FIELD_CELL_OF && field <= PB_FIELD_R_SORTED;
  if (cell_field && !h->cells_ready) return fail(h, PB_ERR_STATE, "no cell list");
  const void *src = nullptr;
  switch (field) {
    case PB_FIELD_R: src = h->r; break;
    case PB_FIELD_V:
      if (!h->v) return fail(h, PB_ERR_STATE, "handle keeps FP64 velocities");
      src = h->v; break;
    case PB_FIELD_VD:
      if (!h->vd) return fail(h, PB_ERR_STATE, "handle keeps FP32 velocities");
      src = h->vd; break;
    case PB_FIELD_F: src = h->F[h->cur]; break;
    case PB_FIELD_FOLD: src = h->F[1 - h->cur]; break;
    case PB_FIELD_MINV: src = h->minv; break;
    case PB_FIELD_MASS: src = h->mass; break;
    case PB_FIELD_TYPE: src = h->type; break;
    case PB_FIELD_PID: src = h->pid; break;
    case PB_FIELD_CELL_START: src = h->start; break;
    case PB_FIELD_R_SORTED: src = h->rs; break;
    case PB_FIELD_CELL_OF: {
      std::vector<uint32_t> k(h->N);
      PB_CUDA(cudaMemcpyAsync(k.data(), h->key, 4 * h->N, cudaMemcpyDeviceToHost, h->stream));
      PB_CUDA(cudaStreamSynchronize(h->stream));
      uint32_t *o = (uint32_t *)host;
      for (uint32_t i = 0; i < h->N; ++i) o[i] = h->ref_of_key[k[i]];
      return PB_OK;
    }
    case PB_FIELD_CELL_KEY:
      std::memcpy(host, h->key_of_ref.data(), need);
      return PB_OK;
    case PB_FIELD_NEIGHBORS: {
      std::vector<uint32_t> t;
      neighbor_table(h->grid, t);
      std::memcpy(host, t.data(), need);
      return PB_OK;
    }
    default: return PB_ERR_NOTFOUND;
  }
  PB_CUDA(cudaMemcpyAsync(host, src, need, cudaMemcpyDeviceToHost, h->stream));
  PB_CUDA(cudaStreamSynchronize(h->stream));
  return PB_OK;
}

int pb_md_set(pb_md *h, int field, const void *host, size_t bytes) {
  if (!h || !host) return PB_ERR_ARG;
  size_t need = 0;
  int rc = pb_md_field_bytes(h, field, &need);
  if (rc) return rc;
  if (bytes != need) return fail(h, PB_ERR_ARG, "size mismatch for field");
  void *dst = nullptr;
  switch (field) {
    case PB_FIELD_R: dst = h->r; break;
    case PB_FIELD_V: dst = h->v; break;
    case PB_FIELD_VD: dst = h->vd; break;
    case PB_FIELD_F: dst = h->F[h->cur]; break;
    case PB_FIELD_FOLD: dst = h->F[1 - h->cur]; break;
    case PB_FIELD_MINV: dst = h->minv; break;
    case PB_FIELD_TYPE: dst = h->type; break;
    default: return fail(h, PB_ERR_ARG, "field is read-only");
  }
  if (!dst) return fail(h, PB_ERR_STATE, "field not allocated for this handle");
  PB_CUDA(cudaMemcpyAsync(dst, host, need, cudaMemcpyHostToDevice, h->stream));
  PB_CUDA(cudaStreamSynchronize(h->stream));
  if (field == PB_FIELD_MINV) {
    std::vector<float> mi(h->N), m(h->N);
    std::memcpy(mi.data(), host, need);
    for (uint32_t i = 0; i < h->N; ++i) m[i] = 1.0f / mi[i];
    PB_CUDA(cudaMemcpyAsync(h->mass, m.data(), need, cudaMemcpyHostToDevice, h->stream));
    PB_CUDA(cudaStreamSynchronize(h->stream));
  }
  return PB_OK;
}

}  // extern "C"
