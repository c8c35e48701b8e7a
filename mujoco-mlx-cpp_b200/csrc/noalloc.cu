// Allocation-free physics step: mjb200_batched_step_noalloc.
//
// Who cannot allocate: a training program that hands all free device memory
// to its own caching allocator at start-up (an RL trainer that reserves the
// GPU for its replay buffers and networks) finds cudaMalloc failing or
// fragmenting its pool; a real-time control loop cannot wait on cudaMalloc /
// cudaFree, which may synchronise the device and take milliseconds; a host
// process that fixes its device-memory budget when it starts may not let a
// library grow it later.  This entry point steps a sim whose state lives in
// the caller's own device buffers and allocates nothing on any call.
//
// Scratch: the step kernel needs a work-queue head (independent-warp launch
// mode) and six per-env statistics arrays.  They live in the file-scope
// device array below, sized for MJB200_NOALLOC_MAX_ENVS envs (about 1.5 MB
// per GPU, part of the library image, held by every GPU that loads the
// library until the process exits).  A sim with more envs is rejected with an
// error; the kernel never reads or writes past the array.
//
// Set-up: in host code the array's name is a host-side stand-in, not a
// device address.  The device address is looked up with cudaGetSymbolAddress
// on the first call made on each device (with that device current) and
// cached; that lookup may initialise the device's CUDA context, so make the
// first call on each device before any stream capture begins.
//
// What must start at zero: only the work-queue head; every call that uses
// the queue clears it on the caller's stream before the launch.  The
// statistics are overwritten by each launch, and the array keeps the last
// call's contents.
//
// Concurrency: the scratch is shared by every sim on the device.  Two calls
// whose kernels overlap on the GPU (different streams, different threads,
// different sims) race on the queue head and the statistics; order them on
// one stream or synchronise between them.
#include <cuda_runtime.h>

#include <mutex>
#include <stdexcept>
#include <string>

#include "capi_internal.h"
#include "engine.h"
#include "step_params.h"

cudaError_t mjb_launch_step(const StepParams& P, int grid, int warps_per_block, size_t smem_bytes, cudaStream_t stream);

#define MJB200_NOALLOC_MAX_ENVS 65536
#define MJB200_NOALLOC_HEAD_WORDS 64  // queue head, padded to 256 bytes

static __device__ __align__(256) int g_mjb200_noalloc_scratch[MJB200_NOALLOC_HEAD_WORDS + 6 * MJB200_NOALLOC_MAX_ENVS];

namespace {

constexpr int kMaxDevices = 64;
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
  if (e == cudaSuccess) {
    // the sim's own launch shape (chosen, and its shared-memory limit set,
    // when the sim was created): the same stage code in the same mapping as
    // the regular step, so the results are the same
    int grid = 1, warps = 1, smem = 0, persistent = 0;
    E.launch_shape(&grid, &warps, &smem, &persistent);
    const bool queue = persistent && !E.lockstep();
    StepParams P = E.external_params(qpos, qvel, ctrl, qacc_warmstart, n, queue ? scratch : nullptr, scratch + MJB200_NOALLOC_HEAD_WORDS);
    P.lockstep = E.lockstep();
    if (queue) e = cudaMemsetAsync(scratch, 0, sizeof(int), s);
    if (e == cudaSuccess) e = mjb_launch_step(P, grid, warps, (size_t)smem, s);
  }
  if (e != cudaSuccess) {
    mjb::set_error(std::string("mjb200_batched_step_noalloc: ") + cudaGetErrorString(e));
    return -3;
  }
  return 0;
}
