#include "engine.h"
#include <atomic>
#include <thread>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>

#include "../../include/pb/pb.h"
#include "plan.h"

namespace pb {
namespace {

int fail(Engine &e, int code, const std::string &msg) {
  e.err = msg;
  return code;
}

int cuda_fail(Engine &e, cudaError_t c, const char *what) {
  return fail(e, PB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(c));
}

#define E_CUDA(call)                                       \
  do {                                                     \
    cudaError_t c_ = (call);                               \
    if (c_ != cudaSuccess) return cuda_fail(e, c_, #call); \
  } while (0)

// Engine memory comes from a stream-ordered pool per device that keeps the
// memory it frees (a caching allocator), so the batches a server builds and
// drops at every repack reuse memory instead of mapping new pages each time.
constexpr uint64_t kPoolKeep = ~0ull;

cudaMemPool_t device_pool() {
  static std::mutex mu;
  static std::map<int, cudaMemPool_t> pools;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  std::lock_guard<std::mutex> lk(mu);
  auto it = pools.find(dev);
  if (it != pools.end()) return it->second;
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = dev;
  cudaMemPool_t pool = nullptr;
  if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) return nullptr;
  uint64_t keep = kPoolKeep;
  cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  pools[dev] = pool;
  return pool;
}

template <typename T>
cudaError_t dalloc(Engine &e, T **p, size_t count) {
  if (count == 0) count = 1;
  cudaMemPool_t pool = device_pool();
  if (!pool) return cudaErrorMemoryAllocation;
  return cudaMallocFromPoolAsync((void **)p, sizeof(T) * count, pool, e.stream);
}

template <typename T>
void dfree(Engine &e, T *&p) {
  if (p) cudaFreeAsync((void *)p, e.stream);
  p = nullptr;
}

}  // namespace

// Scratch of the batch and server paths comes from the same pool: memory from
// CUDA's default pool (release threshold 0) made stream synchronisations
// after a repack stall for hundreds of milliseconds.
cudaError_t engine_alloc_bytes(Engine &e, void **p, size_t bytes) {
  cudaMemPool_t pool = device_pool();
  if (!pool) return cudaErrorMemoryAllocation;
  return cudaMallocFromPoolAsync(p, bytes ? bytes : 1, pool, e.stream);
}

void engine_free_bytes(Engine &e, void *p) {
  if (p) cudaFreeAsync(p, e.stream);
}

// Growing the pool maps new pages.  Inside a running server a growth took
// from a few hundred milliseconds to a second, whatever its size, and a server
// that grew the pool batch by batch spent 8 s of a 2,000-job run in them.  A
// server therefore takes its memory into the pool once, at creation: one block
// of `bytes`, given back at once; the pool keeps what it frees.
int engine_pool_reserve(size_t bytes) {
  if (bytes == 0) return PB_OK;
  cudaMemPool_t pool = device_pool();
  if (!pool) return PB_ERR_CUDA;
  cudaStream_t s = nullptr;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return PB_ERR_CUDA;
  void *p = nullptr;
  int rc = PB_OK;
  uint64_t held = 0;
  cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &held);
  if (cudaMallocFromPoolAsync(&p, bytes, pool, s) == cudaSuccess) {
    cudaFreeAsync(p, s);
  } else {
    cudaGetLastError();  // allocation failures are not sticky
    // a failed growth can leave the pages it did map in the pool: give them back
    cudaMemPoolTrimTo(pool, (size_t)held);
    rc = PB_ERR_OOM;
  }
  if (cudaStreamSynchronize(s) != cudaSuccess) rc = PB_ERR_CUDA;
  cudaStreamDestroy(s);
  return rc;
}

// Hands the pool's unused memory back to the device.
void engine_pool_trim() {
  if (cudaMemPool_t pool = device_pool()) cudaMemPoolTrimTo(pool, 0);
}

namespace {

// Column ranking and force work items depend only on the grid and the z-run
// length; batches of many similar systems share them.
struct PlanKey {
  int nx, ny, nz, seg, periodic;
  bool operator<(const PlanKey &o) const {
    return std::tie(nx, ny, nz, seg, periodic) < std::tie(o.nx, o.ny, o.nz, o.seg, o.periodic);
  }
};
struct Plan {
  std::vector<uint32_t> rank, xy;
  std::vector<ForceItem> items;  // system 0, cell0 0
};

// A plan's tables in device memory (per device, kept for the process): a new
// batch's items and column tables are expanded from them on the device, so a
// repack of ~1,500 systems uploads one record per system instead of ~10 MB
// of items built on the host.
struct DevPlan {
  std::shared_ptr<const Plan> keep;  // the host plan stays alive with its key
  int dev = 0;
  ForceItem *items = nullptr;
  uint32_t *rank = nullptr, *xy = nullptr;
  DevPlan() = default;
  DevPlan(const DevPlan &) = delete;
  DevPlan &operator=(const DevPlan &) = delete;
  ~DevPlan() {  // the last user is done with it (cudaFree waits for the device)
    int cur = 0;
    if (cudaGetDevice(&cur) != cudaSuccess) return;
    cudaSetDevice(dev);
    cudaFree(items);
    cudaFree(rank);
    cudaFree(xy);
    cudaSetDevice(cur);
  }
};

// The cache holds one reference and every engine set-up that uses a plan
// another, so a cache that starts over frees no table still being expanded.
std::shared_ptr<const DevPlan> device_plan(const std::shared_ptr<const Plan> &p) {
  static std::mutex mu;
  static std::map<std::pair<int, const Plan *>, std::shared_ptr<const DevPlan>> cache;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  std::lock_guard<std::mutex> lk(mu);
  const auto key = std::make_pair(dev, p.get());
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  if (cache.size() > 4096) cache.clear();  // many distinct grids: start over
  auto d = std::make_shared<DevPlan>();
  d->keep = p;
  d->dev = dev;
  const size_t ni = std::max<size_t>(1, p->items.size()), nc = std::max<size_t>(1, p->rank.size());
  bool ok = cudaMalloc(&d->items, sizeof(ForceItem) * ni) == cudaSuccess &&
            cudaMalloc(&d->rank, 4 * nc) == cudaSuccess && cudaMalloc(&d->xy, 4 * nc) == cudaSuccess;
  ok = ok &&
       cudaMemcpy(d->items, p->items.data(), sizeof(ForceItem) * p->items.size(),
                  cudaMemcpyHostToDevice) == cudaSuccess &&
       cudaMemcpy(d->rank, p->rank.data(), 4 * p->rank.size(), cudaMemcpyHostToDevice) ==
           cudaSuccess &&
       cudaMemcpy(d->xy, p->xy.data(), 4 * p->xy.size(), cudaMemcpyHostToDevice) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();  // allocation failures are not sticky
    return nullptr;      // d frees what it holds
  }
  cache[key] = d;
  return d;
}

// One system's share of the expansion: its plan's device tables and where its
// items, columns and cells start in the batch.
struct SysPlan {
  const ForceItem *items;
  const uint32_t *rank, *xy;
  uint32_t nitems, ncols, item0, col0, cell0;
};

// Block s writes system s's items (its index, cell keys offset by its first
// cell) and column tables: the same records the host would build.
__global__ void k_expand_plans(const SysPlan *sp, ForceItem *items, uint32_t *rank,
                               uint32_t *xy) {
  const SysPlan P = sp[blockIdx.x];
  for (uint32_t k = threadIdx.x; k < P.nitems; k += blockDim.x) {
    ForceItem it = P.items[k];
    it.sys = blockIdx.x;
#pragma unroll
    for (int c = 0; c < 9; ++c)
      if (it.kbase[c] != kNoCell) it.kbase[c] += P.cell0;
    items[P.item0 + k] = it;
  }
  for (uint32_t k = threadIdx.x; k < P.ncols; k += blockDim.x) {
    rank[P.col0 + k] = P.rank[k];
    xy[P.col0 + k] = P.xy[k];
  }
}

std::shared_ptr<const Plan> cached_plan(const Grid &g, int seg) {
  static std::mutex mu;
  static std::map<PlanKey, std::shared_ptr<const Plan>> cache;
  const PlanKey k{g.n[0], g.n[1], g.n[2], seg, g.periodic};
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(k);
    if (it != cache.end()) return it->second;
  }
  auto p = std::make_shared<Plan>();
  morton_columns(g.n[0], g.n[1], p->rank, p->xy);
  append_items(0, g, seg, 0, p->rank, p->xy, p->items);
  std::lock_guard<std::mutex> lk(mu);
  if (cache.size() > 4096) cache.clear();
  cache[k] = p;
  return p;
}

void free_cells(Engine &e) {
  dfree(e, e.key);
  dfree(e, e.within);
  dfree(e, e.tilesum);
  dfree(e, e.count);
  dfree(e, e.start);
  dfree(e, e.bucket);
  dfree(e, e.ovf);
  dfree(e, e.tcount);
  dfree(e, e.cctl);
  dfree(e, e.pid_tmp);
  dfree(e, e.pid);
  dfree(e, e.slot);
  dfree(e, e.rs);
  dfree(e, e.xs);
  dfree(e, e.ys);
  dfree(e, e.zs);
  dfree(e, e.ts);
  dfree(e, e.colrank);
  dfree(e, e.colxy);
  dfree(e, e.d_sys);
  dfree(e, e.d_items);
  dfree(e, e.d_item0);
  dfree(e, e.fpartials);
  dfree(e, e.fqueue);
  e.cells_ready = false;
}

void free_nlist(Engine &e) {
  dfree(e, e.nl_idx);
  dfree(e, e.nl_cnt);
  dfree(e, e.nl_atom);
  dfree(e, e.nl_max);
  dfree(e, e.nl_r0);
  dfree(e, e.nl_rl);
  dfree(e, e.nl_partials);
  dfree(e, e.d_nl_item0);
  e.nl_cap = 0;
  e.nl_built = false;
}

float max_rc2(const Engine &e) {
  float m = 0.f;
  const LJTable &T = e.sp[0].lj;
  for (int k = 0; k < T.nt * T.nt; ++k) m = std::max(m, T.rc2[k]);
  return m;
}

NlistBufs engine_nbufs(Engine &e) {
  NlistBufs b{};
  b.r = e.r;
  b.rs = e.rs;
  b.pid = e.pid;
  b.start = e.start;
  b.key = e.key;
  b.colxy = e.colxy;
  b.colrank = e.colrank;
  b.type = e.type;
  b.sys = e.d_sys;
  b.lj = e.d_lj;
  b.N = e.N;
  b.cap = e.nl_cap;
  const float rl = std::sqrt(max_rc2(e)) + e.nl_skin;
  b.rl2 = rl * rl;
  b.skin = e.nl_skin;
  b.idx = e.nl_idx;
  b.cnt = e.nl_cnt;
  b.atom = e.nl_atom;
  b.r0 = e.nl_r0;
  b.rl = e.nl_rl;
  b.maxcnt = e.nl_max;
  b.F = e.F[e.cur];
  b.partials = e.nl_partials;
  b.status = e.status;
  return b;
}

}  // namespace

void engine_drop_graph(Engine &e) {
  for (auto &g : e.graph2) {
    if (g) cudaGraphExecDestroy(g);
    g = nullptr;
  }
  for (auto &g : e.graph1) {
    if (g) cudaGraphExecDestroy(g);
    g = nullptr;
  }
  e.graph_mode = -1;
  e.graph_dt.clear();
}

int engine_init(Engine &e, const uint32_t *natoms, uint32_t nsys, uint32_t flags,
                bool zero_state) {
  if (!natoms || nsys == 0) return fail(e, PB_ERR_ARG, "no systems");
  e.flags = flags;
  e.nsys = nsys;
  e.sp.assign(nsys, SysParams{});
  e.atom0.assign(nsys + 1, 0);
  uint64_t total = 0;
  for (uint32_t s = 0; s < nsys; ++s) {
    if (natoms[s] == 0) return fail(e, PB_ERR_ARG, "empty system");
    e.sp[s].n = natoms[s];
    e.atom0[s] = (uint32_t)total;
    total += natoms[s];
  }
  if (total >= (1ull << 31)) return fail(e, PB_ERR_ARG, "too many atoms");
  e.N = (uint32_t)total;
  e.atom0[nsys] = e.N;
  E_CUDA(cudaStreamCreateWithFlags(&e.stream, cudaStreamNonBlocking));
  e.own_stream = true;

  // integration blocks aligned to every system's first atom
  std::vector<uint32_t> blk0(nsys), nblk(nsys);
  e.nblocks = 0;
  for (uint32_t s = 0; s < nsys; ++s) e.nblocks += blocks_for(natoms[s]);
  std::vector<BlockMap> map(e.nblocks);
  make_block_map(natoms, nsys, map.data(), blk0.data(), nblk.data());
  e.sysint.assign(nsys, SysInt{});
  for (uint32_t s = 0; s < nsys; ++s) {
    SysInt &I = e.sysint[s];
    I.atom0 = e.atom0[s];
    I.natoms = natoms[s];
    I.vd0 = 3 * e.atom0[s];
    I.blk0 = blk0[s];
    I.nblk = nblk[s];
    I.dt = e.sp[s].dt;
    for (int k = 0; k < 3; ++k) {
      I.c0[k] = 0.f;
      I.c1[k] = 1.f;
      I.L[k] = 1.f;
    }
  }
  const uint32_t N = e.N;
  bool ok = dalloc(e, &e.r, N) == cudaSuccess && dalloc(e, &e.F[0], N) == cudaSuccess &&
            dalloc(e, &e.F[1], N) == cudaSuccess && dalloc(e, &e.minv, N) == cudaSuccess &&
            dalloc(e, &e.mass, N) == cudaSuccess && dalloc(e, &e.type, N) == cudaSuccess &&
            dalloc(e, &e.d_sysint, nsys) == cudaSuccess && dalloc(e, &e.d_map, e.nblocks) == cudaSuccess &&
            dalloc(e, &e.ipartials, (size_t)8 * e.nblocks) == cudaSuccess &&
            dalloc(e, &e.sc, nsys) == cudaSuccess && dalloc(e, &e.status, nsys) == cudaSuccess &&
            dalloc(e, &e.d_fac, nsys) == cudaSuccess && dalloc(e, &e.d_lj, nsys) == cudaSuccess;
  // the half-shell kernel's fixed-point force sums (48 B/atom), only where it runs
  const bool half = (flags & PB_MD_HALF_SHELL) && !(flags & PB_MD_ACC_FP64);
  if (half) ok = ok && dalloc(e, &e.facc, (size_t)6 * N) == cudaSuccess;
  if (flags & PB_MD_VEL_FP64)
    ok = ok && dalloc(e, &e.vd, (size_t)3 * N) == cudaSuccess;
  else
    ok = ok && dalloc(e, &e.v, N) == cudaSuccess;
  if (nsys > 1) ok = ok && dalloc(e, &e.sysid, N) == cudaSuccess;
  if (!ok) return fail(e, PB_ERR_OOM, "device allocation failed");
  if (zero_state) {
    E_CUDA(cudaMemsetAsync(e.r, 0, sizeof(float4) * N, e.stream));
    E_CUDA(cudaMemsetAsync(e.F[0], 0, sizeof(float4) * N, e.stream));
    E_CUDA(cudaMemsetAsync(e.F[1], 0, sizeof(float4) * N, e.stream));
    if (e.v) E_CUDA(cudaMemsetAsync(e.v, 0, sizeof(float4) * N, e.stream));
    if (e.vd) E_CUDA(cudaMemsetAsync(e.vd, 0, sizeof(double) * 3 * N, e.stream));
    E_CUDA(cudaMemsetAsync(e.type, 0, sizeof(uint16_t) * N, e.stream));
  }
  if (e.facc) E_CUDA(cudaMemsetAsync(e.facc, 0, sizeof(unsigned long long) * 6 * N, e.stream));
  E_CUDA(cudaMemsetAsync(e.sc, 0, sizeof(DevScalars) * nsys, e.stream));
  E_CUDA(cudaMemsetAsync(e.status, 0, sizeof(uint32_t) * nsys, e.stream));
  E_CUDA(cudaMemcpyAsync(e.d_map, map.data(), sizeof(BlockMap) * e.nblocks, cudaMemcpyHostToDevice,
                         e.stream));
  if (e.sysid) E_CUDA(launch_fill_sysid(e.d_map, e.nblocks, e.sysid, e.stream));
  if (const char *t = std::getenv("PB_FORCE_THREADS")) e.force_threads = std::atoi(t);
  int rc = engine_upload_sysint(e);
  if (rc) return rc;
  E_CUDA(cudaStreamSynchronize(e.stream));
  return PB_OK;
}

void engine_free(Engine &e) {
  if (e.stream) cudaStreamSynchronize(e.stream);
  engine_drop_graph(e);
  free_cells(e);
  dfree(e, e.r);
  dfree(e, e.v);
  dfree(e, e.vd);
  dfree(e, e.F[0]);
  dfree(e, e.F[1]);
  dfree(e, e.minv);
  dfree(e, e.mass);
  dfree(e, e.type);
  dfree(e, e.sysid);
  dfree(e, e.d_sysint);
  dfree(e, e.d_map);
  dfree(e, e.ipartials);
  dfree(e, e.sc);
  dfree(e, e.status);
  dfree(e, e.d_fac);
  if (e.h_read) cudaFreeHost(e.h_read);
  e.h_read = nullptr;
  dfree(e, e.facc);
  dfree(e, e.d_lj);
  dfree(e, e.steps_left);
  free_nlist(e);
  if (e.own_stream && e.stream) cudaStreamDestroy(e.stream);
  e.stream = nullptr;
}

int engine_set_stream(Engine &e, cudaStream_t s) {
  E_CUDA(cudaStreamSynchronize(e.stream));
  engine_drop_graph(e);
  if (e.own_stream) cudaStreamDestroy(e.stream);
  e.stream = s;
  e.own_stream = false;
  return PB_OK;
}

int engine_upload_lj(Engine &e) {
  std::vector<LJTable> t(e.nsys);
  for (uint32_t s = 0; s < e.nsys; ++s) t[s] = e.sp[s].lj;
  E_CUDA(cudaMemcpyAsync(e.d_lj, t.data(), sizeof(LJTable) * e.nsys, cudaMemcpyHostToDevice,
                         e.stream));
  E_CUDA(cudaStreamSynchronize(e.stream));
  return PB_OK;
}

int engine_upload_sysint(Engine &e) {
  for (uint32_t s = 0; s < e.nsys; ++s) {
    SysInt &I = e.sysint[s];
    const SysParams &P = e.sp[s];
    I.dt = P.dt;
    for (int k = 0; k < 3; ++k) {
      I.c0[k] = P.cell[2 * k];
      I.c1[k] = P.cell[2 * k + 1];
      I.L[k] = P.cell[2 * k + 1] - P.cell[2 * k];
    }
  }
  E_CUDA(cudaMemcpyAsync(e.d_sysint, e.sysint.data(), sizeof(SysInt) * e.nsys,
                         cudaMemcpyHostToDevice, e.stream));
  E_CUDA(cudaStreamSynchronize(e.stream));
  return PB_OK;
}

void lj_table_fill(SysParams &P, const float *p, uint32_t nt, int stride, bool percut) {
  LJTable &t = P.lj;
  std::memset(&t, 0, sizeof(t));
  t.nt = (int)nt;
  for (uint32_t a = 0; a < nt; ++a)
    for (uint32_t b = 0; b < nt; ++b) {
      const uint32_t k = a * nt + b;
      const float sig = p[stride * k], eps = p[stride * k + 1];
      t.s2[k] = sig * sig;
      t.e24[k] = eps * 24.0f;
      t.e4[k] = eps * 4.0f;
      const float rc2 = percut ? p[stride * k + 2] * p[stride * k + 2] : P.rmax2;
      t.rc2[k] = rc2;
      const double sr6 = rc2 > 0 ? std::pow((double)t.s2[k] / rc2, 3) : 0.0;
      t.ushift[k] = (float)(4.0 * eps * (sr6 * sr6 - sr6));
    }
  P.lj_set = true;
  P.lj_percut = percut;
}

void lj_table_set_rmax2(SysParams &P, float rmax2) {
  P.rmax2 = rmax2;
  if (!P.lj_set || P.lj_percut) return;
  for (int k = 0; k < P.lj.nt * P.lj.nt; ++k) {
    P.lj.rc2[k] = rmax2;
    const double sr6 = std::pow((double)P.lj.s2[k] / rmax2, 3);
    P.lj.ushift[k] = (float)((double)P.lj.e4[k] * (sr6 * sr6 - sr6));
  }
}

void engine_set_dt(Engine &e, float dt) {
  bool changed = false;
  for (auto &P : e.sp) {
    if (P.dt != dt) changed = true;
    P.dt = dt;
  }
  if (changed) engine_upload_sysint(e);
}

// Host conversion of imported atoms runs on several threads over fixed
// chunks; per-chunk mass sums are added in chunk order, so the mean mass does
// not depend on the number of threads.
constexpr uint32_t kImportChunk = 1u << 16;

template <typename F>
void for_chunks(uint32_t n, F &&body) {
  const uint32_t nchunks = (n + kImportChunk - 1) / kImportChunk;
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const unsigned nth = std::min<unsigned>(std::min(hw, 16u), nchunks);
  std::atomic<uint32_t> next{0};
  auto run = [&]() {
    for (uint32_t c; (c = next.fetch_add(1)) < nchunks;)
      body(c, c * kImportChunk, std::min(n, (c + 1) * kImportChunk));
  };
  std::vector<std::thread> th;
  for (unsigned k = 1; k < nth; ++k) th.emplace_back(run);
  run();
  for (auto &t : th) t.join();
}

int engine_import(Engine &e, uint32_t sys, const double *r3, const double *v3, const double *mass,
                  const uint32_t *type) {
  if (sys >= e.nsys || !r3) return fail(e, PB_ERR_ARG, "bad system or positions");
  e.mv2_fresh = false;
  e.sp[sys].r_set = true;
  const uint32_t n = e.sp[sys].n, a0 = e.atom0[sys];
  if (n == 0) return PB_OK;
  std::unique_ptr<float4[]> r4(new float4[n]), v4(e.vd ? nullptr : new float4[n]);
  std::unique_ptr<float[]> minv(new float[n]), m(new float[n]);
  std::unique_ptr<uint16_t[]> t(new uint16_t[n]);
  std::unique_ptr<double[]> vd(e.vd ? new double[(size_t)3 * n] : nullptr);
  const uint32_t nchunks = (n + kImportChunk - 1) / kImportChunk;
  std::vector<double> msum(nchunks, 0.0);
  std::vector<int> bad(nchunks, 0);  // 1: mass, 2: type
  for_chunks(n, [&](uint32_t c, uint32_t i0, uint32_t i1) {
    double ms = 0;
    for (uint32_t i = i0; i < i1; ++i) {
      r4[i] = make_float4((float)r3[3 * i], (float)r3[3 * i + 1], (float)r3[3 * i + 2], 0.f);
      if (v4)
        v4[i] = v3 ? make_float4((float)v3[3 * i], (float)v3[3 * i + 1], (float)v3[3 * i + 2], 0.f)
                   : make_float4(0.f, 0.f, 0.f, 0.f);
      if (vd)
        for (int k = 0; k < 3; ++k) vd[(size_t)k * n + i] = v3 ? v3[3 * i + k] : 0.0;
      const double mi = mass ? mass[i] : 1.0;
      if (!(mi > 0)) bad[c] |= 1;
      minv[i] = (float)(1.0 / mi);  // cudaParticleBase::import: TMP[i] = 1.0 / m
      m[i] = 1.0f / minv[i];        // cudaParticleMD::setM: m = 1 / minv
      ms += mi;
      uint16_t ti = 0;
      if (type) {
        if (type[i] >= (uint32_t)kMaxTypes) bad[c] |= 2;
        ti = (uint16_t)type[i];
      }
      t[i] = ti;
    }
    msum[c] = ms;
  });
  double total = 0;
  int flags = 0;
  for (uint32_t c = 0; c < nchunks; ++c) {
    total += msum[c];
    flags |= bad[c];
  }
  if (flags & 1) return fail(e, PB_ERR_ARG, "mass must be positive");
  if (flags & 2) return fail(e, PB_ERR_ARG, "type id >= 8");
  e.sp[sys].m0 = total / n;
  E_CUDA(cudaMemcpyAsync(e.r + a0, r4.get(), 16 * (size_t)n, cudaMemcpyHostToDevice, e.stream));
  E_CUDA(cudaMemcpyAsync(e.minv + a0, minv.get(), 4 * (size_t)n, cudaMemcpyHostToDevice, e.stream));
  E_CUDA(cudaMemcpyAsync(e.mass + a0, m.get(), 4 * (size_t)n, cudaMemcpyHostToDevice, e.stream));
  E_CUDA(cudaMemcpyAsync(e.type + a0, t.get(), 2 * (size_t)n, cudaMemcpyHostToDevice, e.stream));
  if (e.vd)
    E_CUDA(cudaMemcpyAsync(e.vd + 3 * (size_t)a0, vd.get(), 24 * (size_t)n,
                           cudaMemcpyHostToDevice, e.stream));
  else
    E_CUDA(cudaMemcpyAsync(e.v + a0, v4.get(), 16 * (size_t)n, cudaMemcpyHostToDevice, e.stream));
  E_CUDA(cudaStreamSynchronize(e.stream));
  return PB_OK;
}

// The two cell builds give the same bits.  The bucket build is faster when
// consecutive particles tend to share cells (lattice starts, 1M atoms: 0.042
// against 0.046 ms); the counting sort when the particle order is random
// (8.4M-atom mixture from random positions: 0.59 against 0.83 ms), because the
// bucket build's per-warp aggregation of atomics then finds nothing to merge.
// With positions in place and enough atoms to matter, both run twice on the
// engine's stream and the faster is kept.
void choose_cell_build(Engine &e) {
  if (e.cells_chosen) return;
  e.cells_bucket = true;
  // PB_CELL_BUILD=bucket or sort fixes the choice (tests, measurements)
  if (const char *m = std::getenv("PB_CELL_BUILD")) {
    if (std::strcmp(m, "sort") == 0) e.cells_bucket = false;
    if (std::strcmp(m, "bucket") == 0 || std::strcmp(m, "sort") == 0) return;
  }
  if (e.N < (1u << 16)) return;
  for (const auto &P : e.sp)
    if (!P.r_set) return;
  cudaEvent_t a = nullptr, b = nullptr;
  if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) {
    if (a) cudaEventDestroy(a);
    return;
  }
  float t[2] = {0.f, 0.f};
  bool ok = true;
  for (int rep = 0; rep < 2 && ok; ++rep) {
    for (int k = 0; k < 2 && ok; ++k) {
      e.cells_bucket = k == 0;
      ok = cudaEventRecord(a, e.stream) == cudaSuccess &&
           launch_cell_build(engine_cbufs(e), e.stream) == cudaSuccess &&
           cudaEventRecord(b, e.stream) == cudaSuccess && cudaEventSynchronize(b) == cudaSuccess;
      float ms = 0.f;
      if (ok && cudaEventElapsedTime(&ms, a, b) == cudaSuccess && rep == 1) t[k] = ms;
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  e.cells_bucket = !ok || t[0] <= t[1];
  e.cells_chosen = ok;
}

int engine_setup_cells(Engine &e) {
  e.nl_built = false;  // a list indexes the old sorted slots
  free_cells(e);
  engine_drop_graph(e);
  std::vector<SysDesc> sd(e.nsys);
  e.item0.assign(e.nsys + 1, 0);
  e.cell0.assign(e.nsys + 1, 0);
  uint64_t ncells = 0;
  uint32_t mirror = 0;
  e.cap_max = 0;
  e.cap_half_max = 0;
  double apc_max = 0.0;
  // grids and plans first, then each system's place in the batch
  std::vector<std::shared_ptr<const Plan>> plans(e.nsys);
  for (uint32_t s = 0; s < e.nsys; ++s) {
    SysParams &P = e.sp[s];
    if (!P.cell_set) return fail(e, PB_ERR_STATE, "set the cell first");
    Grid g;
    if (!make_grid(P.cell, P.rmax, g, P.periodic))
      return fail(e, PB_ERR_ARG, "cell grid needs at least 3 cells per axis (blocknum > 2)");
    if (!P.periodic && ((e.flags & PB_MD_HALF_SHELL) || e.nl_on))
      return fail(e, PB_ERR_UNSUPPORTED,
                  "open boundaries run on the full-shell cell-list force only");
    P.grid = g;
    const double apc = (double)P.n / g.ncells;
    apc_max = std::max(apc_max, apc);
    const bool half = (e.flags & PB_MD_HALF_SHELL) && !(e.flags & PB_MD_ACC_FP64);
    P.seg = choose_segment(apc, g.n[2], e.seg_scale, P.lj_set ? P.lj.nt : 1, half);
    P.cap = (uint32_t)choose_capacity(apc, P.seg);
    P.cap_half = (uint32_t)choose_capacity_half(apc, P.seg);
    e.cap_max = std::max(e.cap_max, P.cap);
    e.cap_half_max = std::max(e.cap_half_max, P.cap_half);
    plans[s] = cached_plan(g, P.seg);
  }
  std::vector<SysPlan> spl(e.nsys);
  std::vector<std::shared_ptr<const DevPlan>> dplans(e.nsys);  // held until the expansion is done
  uint64_t nitems = 0, ncols = 0;
  for (uint32_t s = 0; s < e.nsys; ++s) {
    SysParams &P = e.sp[s];
    const Grid g = P.grid;
    const Plan &plan = *plans[s];
    dplans[s] = device_plan(plans[s]);
    const DevPlan *dp = dplans[s].get();
    if (!dp) return fail(e, PB_ERR_OOM, "work item tables");
    const std::vector<uint32_t> &rank = plan.rank;
    e.cell0[s] = (uint32_t)ncells;
    e.item0[s] = (uint32_t)nitems;
    spl[s] = SysPlan{dp->items,
                     dp->rank,
                     dp->xy,
                     (uint32_t)plan.items.size(),
                     (uint32_t)rank.size(),
                     (uint32_t)nitems,
                     (uint32_t)ncols,
                     (uint32_t)ncells};
    P.key_of_ref.clear();
    P.ref_of_key.clear();
    if (e.nsys == 1) {  // reference cell id <-> key, for the single-system getters
      P.key_of_ref.assign(g.ncells, 0);
      P.ref_of_key.assign(g.ncells, 0);
      for (int d0 = 0; d0 < g.n[0]; ++d0)
        for (int d1 = 0; d1 < g.n[1]; ++d1)
          for (int d2 = 0; d2 < g.n[2]; ++d2) {
            const uint32_t ref = d2 + d1 * g.n[2] + d0 * g.n[2] * g.n[1];
            const uint32_t key = rank[d0 * g.n[1] + d1] * g.n[2] + d2;
            P.key_of_ref[ref] = key;
            P.ref_of_key[key] = ref;
          }
    }
    SysDesc &D = sd[s];
    D.g = g;
    D.atom0 = e.atom0[s];
    D.natoms = P.n;
    D.cell0 = (uint32_t)ncells;
    D.col0 = (uint32_t)ncols;
    D.vd0 = 3 * e.atom0[s];
    D.lj = s;
    D.dt = P.dt;
    D.cap = P.cap;
    D.cap_half = P.cap_half;
    D.mirror0 = mirror;
    mirror += (P.n + 3u) & ~3u;
    nitems += plan.items.size();
    ncols += rank.size();
    ncells += g.ncells;
    if (ncells >= 0xffffffffull || nitems >= 0xffffffffull)
      return fail(e, PB_ERR_ARG, "too many cells");
  }
  e.item0[e.nsys] = (uint32_t)nitems;
  e.cell0[e.nsys] = (uint32_t)ncells;
  e.ncells = (uint32_t)ncells;
  e.nitems = (uint32_t)nitems;
  e.mirrorN = mirror + 4u;
  const uint32_t N = e.N, C = e.ncells;
  e.bucket_cap = (uint32_t)choose_bucket_cap(apc_max);
  e.ntile = (C + 63) / 64;
  e.tile_atoms = (uint32_t)choose_tile_atoms(apc_max);
  bool ok = dalloc(e, &e.key, N) == cudaSuccess && dalloc(e, &e.count, C) == cudaSuccess &&
            dalloc(e, &e.start, (size_t)C + 1) == cudaSuccess &&
            dalloc(e, &e.bucket, (size_t)C * e.bucket_cap) == cudaSuccess &&
            dalloc(e, &e.ovf, N) == cudaSuccess &&
            dalloc(e, &e.tcount, e.ntile) == cudaSuccess &&
            dalloc(e, &e.cctl, 2) == cudaSuccess && dalloc(e, &e.pid_tmp, N) == cudaSuccess &&
            dalloc(e, &e.within, N) == cudaSuccess &&
            dalloc(e, &e.tilesum, (C + 4095) / 4096) == cudaSuccess &&
            dalloc(e, &e.pid, N) == cudaSuccess && dalloc(e, &e.slot, N) == cudaSuccess &&
            dalloc(e, &e.rs, N) == cudaSuccess && dalloc(e, &e.xs, e.mirrorN) == cudaSuccess &&
            dalloc(e, &e.ys, e.mirrorN) == cudaSuccess && dalloc(e, &e.zs, e.mirrorN) == cudaSuccess &&
            dalloc(e, &e.ts, e.mirrorN) == cudaSuccess && dalloc(e, &e.colrank, ncols) == cudaSuccess &&
            dalloc(e, &e.colxy, ncols) == cudaSuccess &&
            dalloc(e, &e.d_sys, e.nsys) == cudaSuccess && dalloc(e, &e.d_items, nitems) == cudaSuccess &&
            dalloc(e, &e.d_item0, e.nsys + 1) == cudaSuccess &&
            dalloc(e, &e.fpartials, (size_t)4 * nitems) == cudaSuccess &&
            dalloc(e, &e.fqueue, 2) == cudaSuccess;
  if (!ok) {
    free_cells(e);
    return fail(e, PB_ERR_OOM, "cell list allocation failed");
  }
  E_CUDA(cudaMemsetAsync(e.count, 0, sizeof(uint32_t) * C, e.stream));
  E_CUDA(cudaMemsetAsync(e.tcount, 0, sizeof(uint32_t) * e.ntile, e.stream));
  E_CUDA(cudaMemsetAsync(e.cctl, 0, sizeof(uint32_t) * 2, e.stream));
  E_CUDA(cudaMemsetAsync(e.fqueue, 0, sizeof(uint32_t) * 2, e.stream));
  SysPlan *d_spl = nullptr;
  E_CUDA(engine_alloc_bytes(e, (void **)&d_spl, sizeof(SysPlan) * e.nsys));
  E_CUDA(cudaMemcpyAsync(d_spl, spl.data(), sizeof(SysPlan) * e.nsys, cudaMemcpyHostToDevice,
                         e.stream));
  k_expand_plans<<<e.nsys, 256, 0, e.stream>>>(d_spl, e.d_items, e.colrank, e.colxy);
  E_CUDA(cudaGetLastError());
  engine_free_bytes(e, d_spl);
  E_CUDA(cudaMemcpyAsync(e.d_sys, sd.data(), sizeof(SysDesc) * e.nsys, cudaMemcpyHostToDevice,
                         e.stream));
  E_CUDA(cudaMemcpyAsync(e.d_item0, e.item0.data(), 4 * (size_t)(e.nsys + 1),
                         cudaMemcpyHostToDevice, e.stream));
  E_CUDA(cudaStreamSynchronize(e.stream));
  int rc = engine_upload_lj(e);  // parameters set since the last upload
  if (rc) return rc;
  rc = engine_upload_sysint(e);
  if (rc) return rc;
  choose_cell_build(e);
  e.cells_ready = true;
  return PB_OK;
}

bool engine_ready(const Engine &e) {
  if (!e.cells_ready || e.N == 0) return false;
  for (const auto &P : e.sp)
    if (!P.lj_set) return false;
  return true;
}

IntegrateArgs engine_iargs(Engine &e, int wrap) {
  IntegrateArgs a{};
  a.r = e.r;
  a.v = e.vd ? nullptr : e.v;
  a.vd = e.vd;
  a.F = e.F[e.cur];
  a.Fold = e.F[1 - e.cur];
  a.minv = e.minv;
  a.mass = e.mass;
  a.sys = e.d_sysint;
  a.map = e.d_map;
  a.nblocks = e.nblocks;
  // an open box is never wrapped by a step (pb_md_wrap still wraps on request)
  bool open_box = false;
  for (const auto &P : e.sp) open_box = open_box || !P.periodic;
  a.wrap = wrap && !open_box;
  a.sc = e.sc;
  a.partials = e.ipartials;
  a.status = e.status;
  a.steps_left = e.steps_left;
  return a;
}

CellBufs engine_cbufs(Engine &e) {
  CellBufs b{};
  b.r = e.r;
  b.type = e.type;
  b.sysid = e.nsys > 1 ? e.sysid : nullptr;
  b.sys = e.d_sys;
  b.colrank = e.colrank;
  b.N = e.N;
  b.ncells = e.ncells;
  b.key = e.key;
  b.within = e.within;
  b.tilesum = e.tilesum;
  b.count = e.count;
  b.start = e.start;
  b.pid_tmp = e.pid_tmp;
  b.bucket = e.cells_bucket ? e.bucket : nullptr;
  b.bucket_cap = e.bucket_cap;
  b.ovf = e.ovf;
  b.tcount = e.tcount;
  b.ntile = e.ntile;
  b.tile_atoms = e.tile_atoms;
  b.ctl = e.cctl;
  b.pid = e.pid;
  b.slot = e.slot;
  b.rs = e.rs;
  b.xs = e.xs;
  b.ys = e.ys;
  b.zs = e.zs;
  b.ts = e.ts;
  b.status = e.status;
  return b;
}

ForceBufs engine_fbufs(Engine &e) {
  ForceBufs b{};
  b.rs = e.rs;
  b.xs = e.xs;
  b.ys = e.ys;
  b.zs = e.zs;
  b.ts = e.ts;
  b.start = e.start;
  b.pid = e.pid;
  b.sys = e.d_sys;
  b.colxy = e.colxy;
  b.colrank = e.colrank;
  b.lj = e.d_lj;
  b.items = e.d_items;
  b.nitems = e.nitems;
  b.cap = (int)e.cap_max;
  b.F = e.F[e.cur];
  b.partials = e.fpartials;
  b.queue = e.fqueue;
  b.status = e.status;
  b.steps_left = e.steps_left;
  b.facc = e.facc;
  b.fbig = e.facc ? e.facc + (size_t)3 * e.N : nullptr;
  b.nacc = e.N;
  b.cap_half = (int)e.cap_half_max;
  b.map = e.d_map;
  b.nblocks = e.nblocks;
  b.wait_polls = e.force_wait_polls;
  b.test_flags = e.force_test_flags;
  return b;
}

int engine_build(Engine &e) {
  if (!e.cells_ready) return fail(e, PB_ERR_STATE, "setup_cells first");
  cudaError_t c = launch_cell_build(engine_cbufs(e), e.stream);
  if (c != cudaSuccess) return cuda_fail(e, c, "cell build");
  return PB_OK;
}

int engine_use_nlist(Engine &e, float thickness) {
  if (e.nsys != 1) return fail(e, PB_ERR_UNSUPPORTED, "neighbour lists are per single system");
  engine_drop_graph(e);  // captured steps change with the force path
  if (thickness < 0) {
    e.nl_on = false;
    free_nlist(e);
    return PB_OK;
  }
  if (!(thickness < 1e30f)) return fail(e, PB_ERR_ARG, "bad thickness");
  if (!e.sp[0].periodic)
    return fail(e, PB_ERR_UNSUPPORTED, "the neighbour list needs a periodic box");
  e.nl_on = true;
  e.nl_skin = thickness;
  e.nl_built = false;
  return PB_OK;
}

int engine_make_nlist(Engine &e) {
  if (!e.nl_on) return fail(e, PB_ERR_STATE, "neighbour list not in use");
  if (!engine_ready(e)) return fail(e, PB_ERR_STATE, "need cell, LJ parameters and setup_cells");
  const Grid &g = e.sp[0].grid;
  const float rl = std::sqrt(max_rc2(e)) + e.nl_skin;
  for (int k = 0; k < 3; ++k) {
    // the 27-cell stencil must reach every pair within the list radius, as the
    // reference's cell blocks (setupCutoffBlock(rc + thickness)) do
    if (g.len[k] < rl) return fail(e, PB_ERR_ARG, "cell edge below cutoff + thickness");
  }
  const uint32_t N = e.N;
  if (e.nl_cap == 0) {
    // expected row length at the system's density, with headroom
    const double vol = (double)g.L[0] * g.L[1] * g.L[2];
    const double expect = N / vol * 4.18879020478639 * rl * rl * rl;
    const uint32_t cap = ((uint32_t)(1.5 * expect) + 32u + 7u) & ~7u;
    const uint32_t nb = nlist_blocks(N);
    const uint32_t item0[2] = {0u, nb};
    bool ok = dalloc(e, &e.nl_idx, (size_t)cap * N) == cudaSuccess &&
              dalloc(e, &e.nl_cnt, N) == cudaSuccess && dalloc(e, &e.nl_atom, N) == cudaSuccess &&
              dalloc(e, &e.nl_max, 1) == cudaSuccess && dalloc(e, &e.nl_r0, N) == cudaSuccess &&
              dalloc(e, &e.nl_rl, N) == cudaSuccess &&
              dalloc(e, &e.nl_partials, (size_t)4 * nb) == cudaSuccess &&
              dalloc(e, &e.d_nl_item0, 2) == cudaSuccess;
    if (!ok) {
      free_nlist(e);
      return fail(e, PB_ERR_OOM, "neighbour list allocation failed");
    }
    E_CUDA(cudaMemcpyAsync(e.d_nl_item0, item0, sizeof(item0), cudaMemcpyHostToDevice, e.stream));
    e.nl_cap = cap;
    engine_drop_graph(e);  // captured steps hold the old buffers
  }
  for (int attempt = 0; attempt < 2; ++attempt) {
    int rc = engine_build(e);
    if (rc) return rc;
    E_CUDA(cudaMemsetAsync(e.nl_max, 0, sizeof(uint32_t), e.stream));
    cudaError_t c = launch_nlist_build(engine_nbufs(e), e.stream);
    if (c != cudaSuccess) return cuda_fail(e, c, "list build");
    uint32_t mx = 0;
    E_CUDA(cudaMemcpyAsync(&mx, e.nl_max, sizeof(mx), cudaMemcpyDeviceToHost, e.stream));
    E_CUDA(cudaStreamSynchronize(e.stream));
    if (mx <= e.nl_cap) {
      e.nl_built = true;
      return PB_OK;
    }
    // a row did not fit: grow the rows and build again (the overflow bit the
    // build raised is cleared; the rebuilt list is complete)
    dfree(e, e.nl_idx);
    const uint32_t cap = (mx + mx / 4 + 7u) & ~7u;
    if (dalloc(e, &e.nl_idx, (size_t)cap * N) != cudaSuccess) {
      free_nlist(e);
      return fail(e, PB_ERR_OOM, "neighbour list allocation failed");
    }
    e.nl_cap = cap;
    engine_drop_graph(e);
    std::vector<uint32_t> bits;
    engine_status(e, bits);  // read and clear the overflow bit of the failed build
  }
  return fail(e, PB_ERR_DEVICE, "neighbour list rows still overflow");
}

int engine_nlist_info(Engine &e, double out[3]) {
  if (!e.nl_on || !e.nl_built) return fail(e, PB_ERR_STATE, "no neighbour list");
  std::vector<uint32_t> cnt(e.N);
  E_CUDA(cudaMemcpyAsync(cnt.data(), e.nl_cnt, sizeof(uint32_t) * e.N, cudaMemcpyDeviceToHost,
                         e.stream));
  E_CUDA(cudaStreamSynchronize(e.stream));
  double sum = 0;
  uint32_t mx = 0;
  for (uint32_t v : cnt) {
    sum += v;
    mx = std::max(mx, v);
  }
  out[0] = e.N ? sum / e.N : 0.0;
  out[1] = mx;
  out[2] = e.nl_cap;
  return PB_OK;
}

int engine_gr(Engine &e, float rstep, float rmax, uint64_t *counts, uint32_t *rnum) {
  if (e.nsys != 1) return fail(e, PB_ERR_UNSUPPORTED, "g(r) is per single system");
  if (!(rstep > 0) || !(rmax > 0) || !rnum) return fail(e, PB_ERR_ARG, "bad g(r) bins");
  if (!e.sp[0].cell_set) return fail(e, PB_ERR_STATE, "set the cell first");
  // cudaCalcGR::setup (cudaCalcGR.hh:27-31): rstepinv = 1 / rstep as a double
  // quotient stored in FP32, rnum = trunc(rmax * rstepinv) in FP32
  const float inv = (float)(1.0 / (double)rstep);
  const uint32_t n = (uint32_t)(rmax * inv);
  *rnum = n;
  if (!counts) return PB_OK;
  if (n > gr_max_bins()) return fail(e, PB_ERR_ARG, "more g(r) bins than supported");
  const float *c = e.sp[0].cell;
  const float L[3] = {c[1] - c[0], c[3] - c[2], c[5] - c[4]};
  unsigned long long *d = nullptr;
  if (dalloc(e, &d, n) != cudaSuccess) return fail(e, PB_ERR_OOM, "g(r) counts");
  cudaError_t st = cudaMemsetAsync(d, 0, sizeof(unsigned long long) * n, e.stream);
  if (st == cudaSuccess) st = launch_gr(e.r, e.N, L, inv, n, d, e.stream);
  if (st == cudaSuccess)
    st = cudaMemcpyAsync(counts, d, sizeof(uint64_t) * n, cudaMemcpyDeviceToHost, e.stream);
  dfree(e, d);
  if (st == cudaSuccess) st = cudaStreamSynchronize(e.stream);
  if (st != cudaSuccess) return cuda_fail(e, st, "g(r)");
  return PB_OK;
}

int engine_force(Engine &e, bool energy) {
  if (!engine_ready(e)) return fail(e, PB_ERR_STATE, "need cell, LJ parameters and setup_cells");
  int nt = 1;
  for (const auto &P : e.sp) nt = std::max(nt, P.lj.nt);
  if (e.nl_on) {
    if (!e.nl_built) return fail(e, PB_ERR_STATE, "make the neighbour list first");
    cudaError_t c = launch_nlist_force(engine_nbufs(e), nt, energy,
                                       (e.flags & PB_MD_ACC_FP64) != 0, e.stream);
    if (c != cudaSuccess) return cuda_fail(e, c, "list force");
    e.last = e.cur;
    if (energy) {
      c = launch_energy_total(e.nl_partials, e.d_nl_item0, 1, e.sc, e.stream);
      if (c != cudaSuccess) return cuda_fail(e, c, "energy total");
    }
    e.energy_valid = energy;
    return PB_OK;
  }
  // every ordered pair (the reference's full shell), or with PB_MD_HALF_SHELL
  // every unordered pair once with exact fixed-point sums
  const bool full = (e.flags & PB_MD_ACC_FP64) != 0 || (e.flags & PB_MD_HALF_SHELL) == 0;
  cudaError_t c = full ? launch_force(engine_fbufs(e), nt, energy, (e.flags & PB_MD_ACC_FP64) != 0,
                                      e.force_threads, e.stream)
                       : launch_force_half(engine_fbufs(e), nt, energy, e.stream);
  if (c != cudaSuccess) return cuda_fail(e, c, "force");
  e.last = e.cur;
  if (energy) {
    c = launch_energy_total(e.fpartials, e.d_item0, e.nsys, e.sc, e.stream);
    if (c != cudaSuccess) return cuda_fail(e, c, "energy total");
  }
  e.energy_valid = energy;
  return PB_OK;
}

int engine_evolve(Engine &e, int mode, int wrap) {
  IntegrateArgs a = engine_iargs(e, wrap);
  cudaError_t c;
  if (mode == PB_MODE_VV) {
    if (e.vd) return fail(e, PB_ERR_UNSUPPORTED, "velocity Verlet uses FP32 velocities");
    c = launch_vv(a, e.stream);
  } else {
    c = launch_gauss(a, e.stream);
  }
  if (c != cudaSuccess) return cuda_fail(e, c, "time evolution");
  e.cur = 1 - e.cur;
  ++e.steps_done;
  // k_vv and k_gauss_b end with sum m v^2 of the new velocities, added in the
  // same order as k_mv2, so a temperature read needs no further kernel
  e.mv2_fresh = true;
  return PB_OK;
}

int engine_wrap(Engine &e) {
  cudaError_t c = launch_wrap(engine_iargs(e, 1), e.stream);
  if (c != cudaSuccess) return cuda_fail(e, c, "wrap");
  return PB_OK;
}

int engine_step(Engine &e, int mode) {
  // with a neighbour list the cell list is rebuilt only with the list
  int rc = e.nl_on ? PB_OK : engine_build(e);
  if (!rc) rc = engine_force(e, false);
  if (!rc) rc = engine_evolve(e, mode, 1);
  return rc;
}

int engine_run(Engine &e, int mode, uint32_t steps) {
  if (!engine_ready(e)) return fail(e, PB_ERR_STATE, "need cell, LJ parameters and setup_cells");
  if (mode != PB_MODE_VV && mode != PB_MODE_GAUSS) return fail(e, PB_ERR_ARG, "bad mode");
  if (mode == PB_MODE_VV && e.vd) return fail(e, PB_ERR_UNSUPPORTED, "VV needs FP32 velocities");
  std::vector<float> dts(e.nsys);
  for (uint32_t s = 0; s < e.nsys; ++s) dts[s] = e.sp[s].dt;
  if (e.graph_mode != mode || e.graph_dt != dts) engine_drop_graph(e);
  e.graph_mode = mode;
  e.graph_dt = dts;
  // capture `n` whole steps starting from the current ping-pong parity
  auto capture = [&](int n, cudaGraphExec_t *out) -> int {
    cudaGraph_t g = nullptr;
    const int cur0 = e.cur, last0 = e.last;
    const uint64_t done0 = e.steps_done;
    const bool fresh0 = e.mv2_fresh;
    E_CUDA(cudaStreamBeginCapture(e.stream, cudaStreamCaptureModeThreadLocal));
    int rc = PB_OK;
    for (int k = 0; k < n && !rc; ++k) rc = engine_step(e, mode);
    cudaError_t c = cudaStreamEndCapture(e.stream, &g);
    e.cur = cur0;  // the captured steps have not run yet
    e.last = last0;
    e.steps_done = done0;
    e.mv2_fresh = fresh0;
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (c != cudaSuccess) return cuda_fail(e, c, "graph capture");
    c = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (c != cudaSuccess) {
      *out = nullptr;
      return cuda_fail(e, c, "graph instantiate");
    }
    return PB_OK;
  };
  uint32_t done = 0;
  if (steps >= 2) {
    cudaGraphExec_t &g2 = e.graph2[e.cur];  // two steps return to this parity
    if (!g2) {
      const int rc = capture(2, &g2);
      if (rc) return rc;
    }
    for (; done + 2 <= steps; done += 2) {
      E_CUDA(cudaGraphLaunch(g2, e.stream));
      e.steps_done += 2;
      e.last = 1 - e.cur;  // two steps: cur is back where it was, F[1 - cur] is the newest
    }
  }
  if (done < steps) {  // one step left: the one-step graph of this parity
    cudaGraphExec_t &g1 = e.graph1[e.cur];
    if (!g1) {
      const int rc = capture(1, &g1);
      if (rc) return rc;
    }
    E_CUDA(cudaGraphLaunch(g1, e.stream));
    e.steps_done += 1;
    e.last = e.cur;
    e.cur = 1 - e.cur;
  }
  if (steps > 0) e.mv2_fresh = true;  // each step ends with sum m v^2
  e.energy_valid = false;
  return PB_OK;
}

int engine_profile(Engine &e, int mode, uint32_t steps, double ms[3]) {
  if (!engine_ready(e) || steps == 0) return fail(e, PB_ERR_STATE, "not ready");
  cudaEvent_t ev[4];
  for (auto &x : ev) E_CUDA(cudaEventCreate(&x));
  double acc[3] = {0, 0, 0};
  int rc = PB_OK;
  for (uint32_t k = 0; k < steps && !rc; ++k) {
    cudaEventRecord(ev[0], e.stream);
    rc = e.nl_on ? PB_OK : engine_build(e);
    cudaEventRecord(ev[1], e.stream);
    if (!rc) rc = engine_force(e, false);
    cudaEventRecord(ev[2], e.stream);
    if (!rc) rc = engine_evolve(e, mode, 1);
    cudaEventRecord(ev[3], e.stream);
    cudaEventSynchronize(ev[3]);
    for (int p = 0; p < 3; ++p) {
      float t = 0;
      cudaEventElapsedTime(&t, ev[p], ev[p + 1]);
      acc[p] += t;
    }
  }
  for (auto &x : ev) cudaEventDestroy(x);
  for (int p = 0; p < 3; ++p) ms[p] = acc[p] / steps;
  return rc;
}

int engine_set_steps_left(Engine &e, const uint32_t *steps) {
  if (!steps) {
    if (e.steps_left) {
      E_CUDA(cudaStreamSynchronize(e.stream));
      dfree(e, e.steps_left);
      engine_drop_graph(e);  // captured launches hold the old pointer
    }
    return PB_OK;
  }
  if (!e.steps_left) {
    if (dalloc(e, &e.steps_left, e.nsys) != cudaSuccess) return fail(e, PB_ERR_OOM, "steps_left");
    engine_drop_graph(e);  // captured launches hold the old (null) pointer
  }
  e.budget_set.assign(e.nsys, e.steps_done);
  e.budget_end.resize(e.nsys);
  e.last_at_set.assign(e.nsys, e.last);
  for (uint32_t s = 0; s < e.nsys; ++s) e.budget_end[s] = e.steps_done + steps[s];
  E_CUDA(cudaMemcpyAsync(e.steps_left, steps, 4 * (size_t)e.nsys, cudaMemcpyHostToDevice, e.stream));
  E_CUDA(cudaStreamSynchronize(e.stream));
  return PB_OK;
}

int engine_get_steps_left(Engine &e, uint32_t *steps) {
  if (!e.steps_left) return fail(e, PB_ERR_STATE, "no step budgets set");
  E_CUDA(cudaMemcpyAsync(steps, e.steps_left, 4 * (size_t)e.nsys, cudaMemcpyDeviceToHost, e.stream));
  E_CUDA(cudaStreamSynchronize(e.stream));
  return PB_OK;
}

bool engine_finished(const Engine &e, uint32_t s) {
  return e.steps_left && s < e.budget_end.size() && e.steps_done >= e.budget_end[s];
}

int engine_force_buffer(const Engine &e, uint32_t s) {
  if (!engine_finished(e, s)) return e.last;
  if (e.budget_end[s] == e.budget_set[s]) return e.last_at_set[s];  // never ran under this budget
  // its last step was step j = budget_end - 1; step j's force went to the buffer
  // that was `cur` then, and cur flips every step
  const uint64_t back = e.steps_done - (e.budget_end[s] - 1);
  return (back & 1) ? 1 - e.cur : e.cur;
}

int engine_clear_force(Engine &e) {
  E_CUDA(cudaMemsetAsync(e.F[0], 0, sizeof(float4) * e.N, e.stream));
  E_CUDA(cudaMemsetAsync(e.F[1], 0, sizeof(float4) * e.N, e.stream));
  return PB_OK;
}

int engine_mv2(Engine &e) {
  cudaError_t c = launch_mv2(engine_iargs(e, 0), e.stream);
  if (c != cudaSuccess) return cuda_fail(e, c, "mv2");
  e.mv2_fresh = true;
  return PB_OK;
}

int engine_fv(Engine &e) {
  cudaError_t c = launch_fv(engine_iargs(e, 0), e.stream);
  if (c != cudaSuccess) return cuda_fail(e, c, "fv");
  return PB_OK;
}

int engine_scale(Engine &e, const double *factors) {
  e.mv2_fresh = false;
  E_CUDA(cudaMemcpyAsync(e.d_fac, factors, sizeof(double) * e.nsys, cudaMemcpyHostToDevice,
                         e.stream));
  cudaError_t c = launch_scale(engine_iargs(e, 0), e.d_fac, e.stream);
  if (c != cudaSuccess) return cuda_fail(e, c, "scale");
  E_CUDA(cudaStreamSynchronize(e.stream));
  return PB_OK;
}

int engine_adjust(Engine &e, const double *v1) {
  e.mv2_fresh = false;
  E_CUDA(cudaMemcpyAsync(e.d_fac, v1, sizeof(double) * e.nsys, cudaMemcpyHostToDevice, e.stream));
  cudaError_t c = launch_adjust(engine_iargs(e, 0), e.d_fac, e.stream);
  if (c != cudaSuccess) return cuda_fail(e, c, "adjust");
  E_CUDA(cudaStreamSynchronize(e.stream));
  return PB_OK;
}

int engine_force_softcore(Engine &e, float rc, float f0) {
  if (!engine_ready(e)) return fail(e, PB_ERR_STATE, "need cell, LJ parameters and setup_cells");
  if (!(rc > 0)) return fail(e, PB_ERR_ARG, "soft-core range must be > 0");
  int nt = 1;
  for (const auto &P : e.sp) nt = std::max(nt, P.lj.nt);
  ForceBufs b = engine_fbufs(e);
  b.sc_rc = rc;
  b.sc_f0 = f0;
  cudaError_t c = launch_force_softcore(b, nt, e.stream);
  if (c != cudaSuccess) return cuda_fail(e, c, "soft-core force");
  e.last = e.cur;
  e.energy_valid = false;
  return PB_OK;
}

int engine_euler(Engine &e, float dt) {
  e.mv2_fresh = false;
  if (!e.v) return fail(e, PB_ERR_UNSUPPORTED, "the Euler step uses FP32 velocities");
  cudaError_t c = launch_euler(engine_iargs(e, 1), e.F[e.last], dt, e.stream);
  if (c != cudaSuccess) return cuda_fail(e, c, "Euler step");
  return PB_OK;
}

int engine_minimize(Engine &e, uint32_t iters, float alpha, float max_disp) {
  if (!engine_ready(e)) return fail(e, PB_ERR_STATE, "need cell, LJ parameters and setup_cells");
  if (!(alpha > 0) || !(max_disp > 0)) return fail(e, PB_ERR_ARG, "alpha and max_disp must be > 0");
  int nt = 1;
  for (const auto &P : e.sp) nt = std::max(nt, P.lj.nt);
  for (uint32_t it = 0; it < iters; ++it) {
    int rc = engine_build(e);
    if (rc) return rc;
    cudaError_t c = launch_force_capped(engine_fbufs(e), nt, e.stream);
    if (c != cudaSuccess) return cuda_fail(e, c, "relaxation force");
    e.last = e.cur;
    c = launch_sd_move(engine_iargs(e, 1), e.F[e.cur], alpha, max_disp, e.stream);
    if (c != cudaSuccess) return cuda_fail(e, c, "steepest descent");
  }
  e.energy_valid = false;
  E_CUDA(cudaStreamSynchronize(e.stream));
  return PB_OK;
}

int engine_correct_force(Engine &e, const double *lambda) {
  E_CUDA(cudaMemcpyAsync(e.d_fac, lambda, sizeof(double) * e.nsys, cudaMemcpyHostToDevice,
                         e.stream));
  cudaError_t c = launch_correct_force(engine_iargs(e, 0), e.F[e.last], e.d_fac, e.stream);
  if (c != cudaSuccess) return cuda_fail(e, c, "correct force");
  E_CUDA(cudaStreamSynchronize(e.stream));
  return PB_OK;
}

int engine_set_xi(Engine &e, const double *xi) {
  for (uint32_t s = 0; s < e.nsys; ++s)
    E_CUDA(cudaMemcpyAsync(&e.sc[s].xi_old, &xi[s], sizeof(double), cudaMemcpyHostToDevice,
                           e.stream));
  E_CUDA(cudaStreamSynchronize(e.stream));
  return PB_OK;
}

int engine_scalars(Engine &e, std::vector<DevScalars> &out) {
  out.resize(e.nsys);
  E_CUDA(cudaMemcpyAsync(out.data(), e.sc, sizeof(DevScalars) * e.nsys, cudaMemcpyDeviceToHost,
                         e.stream));
  E_CUDA(cudaStreamSynchronize(e.stream));
  return PB_OK;
}

int engine_status(Engine &e, std::vector<uint32_t> &bits) {
  bits.resize(e.nsys);
  E_CUDA(cudaMemcpyAsync(bits.data(), e.status, 4 * (size_t)e.nsys, cudaMemcpyDeviceToHost,
                         e.stream));
  E_CUDA(cudaStreamSynchronize(e.stream));
  E_CUDA(cudaMemsetAsync(e.status, 0, 4 * (size_t)e.nsys, e.stream));
  return PB_OK;
}

}  // namespace pb
