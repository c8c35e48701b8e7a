// Allocation-free physics step: mjb200_batched_step_noalloc.
//
// Some callers cannot let a library allocate device memory while they step:
// code that records the step into a CUDA graph with stream capture (an
// allocation inside the capture region fails or ends the capture), programs
// that reserve their whole device memory budget up front, and real-time
// control loops that must not wait on the allocator.  This entry point lets
// them step a sim whose state lives in their own buffers, and allocates
// nothing on any call.
//
// Scratch: the kernel's variant with the persistent work queue needs a queue
// head and six per-env statistics arrays.  They live in the file-scope device
// array below, sized for MJB200_NOALLOC_MAX_ENVS envs (about 1.5 MB per GPU,
// part of the library image, held until the process exits).  A sim with more
// envs is rejected with an error; it never reads or writes past the array.
//
// Set-up: the array's device address is looked up with cudaGetSymbolAddress
// once per device, on the first call made on that device, and cached.  That
// first lookup may initialise the CUDA context, so make the first call on
// each device before any stream capture begins.
//
// What must start at zero: only the work-queue head; every call clears it on
// the caller's stream before the launch.  The statistics are overwritten by
// each launch.
//
// Concurrency: the scratch is shared by every sim on the device.  Two calls
// whose kernels overlap (different streams, different threads, different
// sims) race on the queue head and the statistics; order them on one stream
// or synchronise between them.
#include <cuda_runtime.h>

#include <mutex>
#include <stdexcept>
#include <string>

#include "capi_internal.h"
#include "engine.h"
#include "step_params.h"

cudaError_t mjb_launch_step(const StepParams& P, int grid, int warps_per_block, size_t smem_bytes, cudaStream_t stream);
cudaError_t mjb_occupancy(int warps_per_block, size_t smem_bytes, int convex, int* blocks_per_sm);

#define MJB200_NOALLOC_MAX_ENVS 65536
#define MJB200_NOALLOC_HEAD_WORDS 64  // queue head, padded to 256 bytes

static __device__ __align__(256) int g_mjb200_noalloc_scratch[MJB200_NOALLOC_HEAD_WORDS + 6 * MJB200_NOALLOC_MAX_ENVS];

namespace {

constexpr int kMaxDevices = 64;
constexpr int kWarpsPerBlock = 4;
std::mutex g_scratch_mutex;
int* g_scratch_addr[kMaxDevices] = {};

cudaError_t scratch_address(int** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_mjb200_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_addr[dev] = static_cast<int*>(p);
  }
  *out = g_scratch_addr[dev];
  return cudaSuccess;
}

}  // namespace

extern "C" MJMLX_API int mjb200_batched_step_noalloc(MjmlxBatchedSim* sim, float* qpos, float* qvel, const float* ctrl, float* qacc_warmstart, int n,
                                                     void* stream) {
  if (!sim || !sim->engine || !qpos || !qvel || !qacc_warmstart || n < 0) {
    mjb::set_error("mjb200_batched_step_noalloc: bad arguments");
    return -1;
  }
  mjb::Engine& E = *sim->engine;
  if (E.total_u() > 0 && !ctrl) {
    mjb::set_error("mjb200_batched_step_noalloc: ctrl is NULL but the model has actuators");
    return -1;
  }
  if (E.num_envs() > MJB200_NOALLOC_MAX_ENVS) {
    mjb::set_error("mjb200_batched_step_noalloc: the sim has " + std::to_string(E.num_envs()) +
                   " envs; the allocation-free step supports at most 65536 (MJB200_NOALLOC_MAX_ENVS)");
    return -2;
  }
  if (E.hbm_workspace()) {
    mjb::set_error("mjb200_batched_step_noalloc: the model's workspace does not fit shared memory (it needs the HBM workspace of the regular step)");
    return -1;
  }
  if (n == 0) return 0;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int* scratch = nullptr;
  cudaError_t e = scratch_address(&scratch);
  const size_t smem = (size_t)kWarpsPerBlock * (E.desc_words() + E.ws_stride()) * 4;
  int bps = 0;
  if (e == cudaSuccess) e = mjb_occupancy(kWarpsPerBlock, smem, E.convex() ? 1 : 0, &bps);
  if (e == cudaSuccess && bps < 1) e = cudaErrorInvalidConfiguration;
  if (e == cudaSuccess) e = cudaMemsetAsync(scratch, 0, sizeof(int), s);
  if (e == cudaSuccess) {
    const int groups = (E.num_envs() + kWarpsPerBlock - 1) / kWarpsPerBlock;
    int grid = E.sm_count() * bps;
    if (grid > groups) grid = groups;
    if (grid < 1) grid = 1;
    StepParams P = E.external_params(qpos, qvel, ctrl, qacc_warmstart, n, scratch, scratch + MJB200_NOALLOC_HEAD_WORDS);
    e = mjb_launch_step(P, grid, kWarpsPerBlock, smem, s);
  }
  if (e != cudaSuccess) {
    mjb::set_error(std::string("mjb200_batched_step_noalloc: ") + cudaGetErrorString(e));
    return -3;
  }
  return 0;
}
