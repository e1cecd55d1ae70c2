// pg_step_static: stepping that allocates nothing.
//
// pg_step draws its per-tile scratch (contacts, constraint rows, island
// buffers) from a buffer the handle cudaMalloc'd. Some callers cannot let a
// call allocate device memory: code running while another component owns
// the device memory (a caching allocator that has reserved it all, or a
// fixed memory budget), latency-critical control loops that must not enter
// the allocator, and callers that have already run out of memory and still
// need to advance the simulation. For them this entry point takes its
// scratch from a fixed array in the library's device image instead.
//
// The array is PG_STATIC_SCRATCH_BYTES (16 MiB) per GPU that loads the
// library, held until the process exits. A call steps as many envs at once
// as fit in it (16 MiB / per-tile scratch) and loops over the rest, so it is
// slower than pg_step on large batches; a model whose per-tile scratch alone
// exceeds the array is rejected. All calls share the array and keep its last
// contents: calls whose work overlaps on the GPU (two handles or two streams
// stepping at the same time on one device) race on it.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "../../include/pippin_b200.h"
#include "../../include/pippin_b200_tools.h"
#include "pg_kernels.h"
#include "pg_model.h"

namespace pg {
// fills the launch arguments of pg_step for [start, end) (pg_api.cpp)
int internal_step_args(pg_handle* h, int64_t start, int64_t end, int64_t nstep, StepArgs* a, SubstepCfg* cfg,
                       cudaStream_t* stream, int* device);
void internal_set_error(const std::string& msg);
}  // namespace pg

namespace {

constexpr size_t PG_STATIC_SCRATCH_BYTES = size_t(16) << 20;
constexpr size_t PG_STATIC_COUNTER_BYTES = 256;  // phase work counters, then tile scratch
// pg_step's scratch buffer ends 64 bytes past its last tile; the static
// tiles leave the same tail free at the array's end
constexpr size_t PG_STATIC_TAIL_BYTES = 64;

// Device-side scratch shared by every pg_step_static call on a device. Host
// code must not use this name as an address: its device address comes from
// cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_static_scratch[PG_STATIC_SCRATCH_BYTES];

// The array's device address on the current device. Looked up on every call
// (the lookup allocates nothing and is cheap), so that a context torn down
// and made again by the host program (cudaDeviceReset) is followed; the
// first lookup on a device loads the library's device image there.
int scratch_address(unsigned char** out) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
  if (e != cudaSuccess) {
    pg::internal_set_error(std::string("cudaGetSymbolAddress(static scratch): ") + cudaGetErrorString(e));
    return PG_ERR_CUDA;
  }
  *out = static_cast<unsigned char*>(p);
  return PG_OK;
}

}  // namespace

extern "C" int pg_static_tiles(size_t tile_bytes, int tiles_per_block, int64_t* tiles) {
  if (!tiles || tile_bytes == 0 || tiles_per_block <= 0) {
    pg::internal_set_error("pg_static_tiles: invalid argument");
    return PG_ERR_INVALID;
  }
  const size_t usable = PG_STATIC_SCRATCH_BYTES - PG_STATIC_COUNTER_BYTES - PG_STATIC_TAIL_BYTES;
  size_t n = usable / tile_bytes;
  *tiles = 0;
  if (n < (size_t)tiles_per_block) {
    pg::internal_set_error("pg_step_static: this model needs " + std::to_string(tile_bytes * tiles_per_block) +
                           " bytes of scratch per block, more than the " + std::to_string(usable) +
                           "-byte static scratch holds (use pg_step)");
    return PG_ERR_UNSUPPORTED;
  }
  *tiles = (int64_t)(n / tiles_per_block * tiles_per_block);
  return PG_OK;
}

extern "C" int pg_step_static(pg_handle* h, int64_t start, int64_t end, int64_t nstep) {
  pg::StepArgs a;
  pg::SubstepCfg cfg;
  cudaStream_t stream;
  int device = 0;
  int rc = pg::internal_step_args(h, start, end, nstep, &a, &cfg, &stream, &device);
  if (rc != PG_OK) return rc;
  if (end == start || nstep == 0) return PG_OK;
  unsigned char* base = nullptr;  // internal_step_args made the handle's device current
  if ((rc = scratch_address(&base)) != PG_OK) return rc;
  // only the Newton phase uses tile scratch: its grid is capped by the array
  pg::LaunchCfg& nc = cfg.newton;
  int64_t tiles = 0;
  if ((rc = pg_static_tiles((size_t)a.s.stride * sizeof(double), nc.tiles_per_block, &tiles)) != PG_OK) return rc;
  nc.blocks = (int)std::min<int64_t>((int64_t)nc.blocks, tiles / nc.tiles_per_block);
  a.queue = reinterpret_cast<int*>(base);
  a.order = nullptr;  // envs in index order: an order array would need memory per env
  a.learn.count = a.queue + pg::Q_LEARN;
  a.scratch = reinterpret_cast<double*>(base + PG_STATIC_COUNTER_BYTES);
  // each substep restarts the phase counters before its kernels
  cudaError_t e = cudaSuccess;
  for (int64_t k = 0; k < nstep && e == cudaSuccess; k++) {
    a.sidx = (int)k;
    e = pg::launch_substep(a, cfg, stream);
  }
  if (e != cudaSuccess) {
    pg::internal_set_error(std::string("pg_step_static: ") + cudaGetErrorString(e));
    return PG_ERR_CUDA;
  }
  return PG_OK;
}
