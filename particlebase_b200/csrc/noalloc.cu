// Cell-list build that allocates no device memory.
//
// The regular path (pb_md_build_cells) keeps its scratch arrays -- per-atom
// cell keys and tickets, per-cell counts, the unordered member list and the
// scan partials -- in buffers the pb_md handle allocates with cudaMalloc.
// Some callers cannot allocate: a host framework that owns every byte of
// device memory through its own pool, or code that must not allocate inside a
// latency-critical loop.  pb_cells_build_noalloc gives them the same build
// with all scratch in one file-scope __device__ array of fixed size, resident
// on every device that loads this library until the process exits.  The
// caller passes the inputs and the outputs; nothing here calls cudaMalloc,
// cudaFree or an allocating library routine.
//
// Limits: at most kMaxAtoms atoms and kMaxCells cells per call (larger sizes
// are rejected with PB_ERR_ARG before any device work).  All calls share the
// one scratch array, so calls that overlap on the GPU (different streams, or
// different host threads) race; serialise them.  The per-cell counters are
// cleared at the start of every call.
//
// The call is stream-ordered and returns without waiting for the GPU: the
// system descriptor and the column ranks travel to the scratch array as
// kernel parameters (copied at launch), so no host memory of the call is read
// after it returns.  The scratch array's device address is resolved once per
// device (cudaGetSymbolAddress) and cached; that address belongs to the
// context the first call ran in, so use one context per device (the primary
// context, as the CUDA runtime does) and do not reset the device between calls.
#include <algorithm>
#include <mutex>
#include <vector>

#include "../../include/pb/pb.h"
#include "md.cuh"
#include "plan.h"

namespace pb {
namespace {

constexpr uint32_t kMaxAtoms = 1u << 17;   // 131,072 atoms
constexpr uint32_t kMaxCells = 1u << 16;   // 65,536 cells
constexpr uint32_t kMaxTiles = (kMaxCells + 4095) / 4096;

// Scratch layout, in order; every block starts on a 256-byte boundary.
struct ScratchLayout {
  uint32_t key[kMaxAtoms];
  uint32_t within[kMaxAtoms];
  uint32_t pid_tmp[kMaxAtoms];
  uint16_t type0[kMaxAtoms];          // zero types when the caller passes none
  uint32_t count[kMaxCells];
  uint32_t colrank[kMaxCells];
  uint32_t tilesum[(kMaxTiles + 63) / 64 * 64];
  SysDesc sys;
};

static __device__ __align__(256) unsigned char g_scratch[sizeof(ScratchLayout)];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void *g_addr[kMaxDevices] = {};

// Device address of g_scratch on the current device, resolved once per
// device.  In host code `g_scratch` names a host-side stand-in, not device
// memory, so the kernels are always given this resolved address.
cudaError_t scratch_on_current_device(ScratchLayout **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_addr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess) return e;
    g_addr[dev] = p;
  }
  *out = reinterpret_cast<ScratchLayout *>(g_addr[dev]);
  return cudaSuccess;
}

// Host values handed to the GPU as kernel parameters: up to kChunk column
// ranks per launch (16 KB of parameters, well inside the 32 KB launch limit),
// and the system descriptor.
constexpr uint32_t kChunk = 4096;
struct RankChunk {
  uint32_t first, n;
  uint32_t v[kChunk];
};

__global__ void k_put_ranks(const RankChunk c, uint32_t *dst) {
  for (uint32_t i = threadIdx.x; i < c.n; i += blockDim.x) dst[c.first + i] = c.v[i];
}

__global__ void k_put_sys(const SysDesc sd, SysDesc *dst) { *dst = sd; }

}  // namespace
}  // namespace pb

using namespace pb;

extern "C" int pb_cells_build_noalloc_limits(uint32_t *max_atoms, uint32_t *max_cells,
                                             size_t *scratch_bytes) {
  if (max_atoms) *max_atoms = kMaxAtoms;
  if (max_cells) *max_cells = kMaxCells;
  if (scratch_bytes) *scratch_bytes = sizeof(ScratchLayout);
  return PB_OK;
}

extern "C" int pb_cells_build_noalloc(const void *r4, const uint16_t *type, uint32_t n,
                                      const float cell6[6], float rmax, uint32_t *start,
                                      uint32_t *pid, uint32_t *slot, void *rs4, void *stream) {
  if (!r4 || !cell6 || !start || !pid || !slot || !rs4 || n == 0) return PB_ERR_ARG;
  if (n > kMaxAtoms) return PB_ERR_ARG;
  Grid g;
  if (!make_grid(cell6, rmax, g)) return PB_ERR_ARG;
  if (g.ncells > kMaxCells) return PB_ERR_ARG;
  ScratchLayout *sc = nullptr;
  if (scratch_on_current_device(&sc) != cudaSuccess) return PB_ERR_CUDA;
  cudaStream_t s = (cudaStream_t)stream;

  // Host-side tables: system descriptor and Z-order column ranks, written
  // into the static scratch by kernels that carry them as parameters.
  std::vector<uint32_t> rank, xy;
  morton_columns(g.n[0], g.n[1], rank, xy);
  SysDesc sd{};
  sd.g = g;
  sd.natoms = n;
  k_put_sys<<<1, 1, 0, s>>>(sd, &sc->sys);
  if (cudaGetLastError() != cudaSuccess) return PB_ERR_CUDA;
  {
    RankChunk c;  // ~16 KB on the host stack, copied into the launch
    for (uint32_t first = 0; first < (uint32_t)rank.size(); first += kChunk) {
      c.first = first;
      c.n = std::min<uint32_t>(kChunk, (uint32_t)rank.size() - first);
      std::copy(rank.begin() + first, rank.begin() + first + c.n, c.v);
      k_put_ranks<<<1, 256, 0, s>>>(c, sc->colrank);
      if (cudaGetLastError() != cudaSuccess) return PB_ERR_CUDA;
    }
  }
  if (cudaMemsetAsync(sc->count, 0, sizeof(uint32_t) * g.ncells, s) != cudaSuccess)
    return PB_ERR_CUDA;
  if (!type && cudaMemsetAsync(sc->type0, 0, sizeof(uint16_t) * n, s) != cudaSuccess)
    return PB_ERR_CUDA;

  CellBufs b{};
  b.r = reinterpret_cast<const float4 *>(r4);
  b.type = type ? type : sc->type0;
  b.sysid = nullptr;
  b.sys = &sc->sys;
  b.colrank = sc->colrank;
  b.N = n;
  b.ncells = g.ncells;
  b.key = sc->key;
  b.within = sc->within;
  b.count = sc->count;
  b.start = start;
  b.tilesum = sc->tilesum;
  b.pid_tmp = sc->pid_tmp;
  b.pid = pid;
  b.slot = slot;
  b.rs = reinterpret_cast<float4 *>(rs4);
  b.status = nullptr;
  if (launch_cell_build(b, s) != cudaSuccess) return PB_ERR_CUDA;
  return PB_OK;
}
