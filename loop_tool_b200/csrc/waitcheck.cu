// Self-check of the bounded waits: runs the give-up path that every
// mbarrier wait in these kernels has (csrc/async.cuh), on a wait that
// cannot complete, with a caller-chosen short limit.
//
// One CTA of one warp, shaped like the tensor-core kernels' wind-down:
//   1. warp 0 allocates TMEM (32 columns) and gives up its allocation permit;
//   2. lane 0 starts one 256-byte bulk copy global -> shared that completes
//      on mbarrier `landed` (a copy in flight, as in a running pipeline);
//   3. lane 0 waits on mbarrier `never`, which nothing arrives at, for at
//      most `limit` cycles: the wait gives up and raises the stream's
//      timeout flag;
//   4. lane 0 waits (bounded, ignoring the flag) for its copy to land;
//   5. warp 0 frees the TMEM and the kernel returns.
// The host then synchronises the stream and reads the flag: the check
// passes when the call reports LTB_ERR_TIMEOUT, and a tensor-core launch
// after it (which allocates TMEM on the same SMs) still runs.
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/loop_tool_b200.h"
#include "async.cuh"
#include "kernels.h"

namespace {

// source of the in-flight copy (16-byte aligned, never written), and the
// check's record: {wait completed, copy drained}
__device__ __align__(16) float g_wait_src[64];
__device__ int g_wait_status[2];

__global__ void __launch_bounds__(32) k_wait_check(int* err, long long limit) {
  __shared__ __align__(128) float dst[64];
  __shared__ __align__(8) uint64_t landed, never;
  __shared__ uint32_t tmem_slot;
  const int lane = threadIdx.x;
  if (lane == 0) {
    mbar_init(smem_u32(&landed), 1);
    mbar_init(smem_u32(&never), 1);
    fence_mbar_init();
  }
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(&tmem_slot)),
               "r"(32));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncwarp();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;
  if (lane == 0) {
    mbar_expect_tx(smem_u32(&landed), (uint32_t)sizeof(dst));
    bulk_load(smem_u32(dst), g_wait_src, (uint32_t)sizeof(dst), smem_u32(&landed));
    const bool completed = mbar_wait_for(smem_u32(&never), 0u, err, limit);
    const bool drained = mbar_drain(smem_u32(&landed), 0u);
    g_wait_status[0] = completed ? 1 : 0;
    g_wait_status[1] = drained ? 1 : 0;
  }
  __syncwarp();
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(32));
}

}  // namespace

// Launches the check on st and copies its record to status_host[2]
// (stream-ordered; complete once st is).
cudaError_t ltb_launch_wait_check(int* err, long long limit, int* status_host, cudaStream_t st) {
  k_wait_check<<<1, 32, 0, st>>>(err, limit);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return cudaMemcpyFromSymbolAsync(status_host, g_wait_status, 2 * sizeof(int), 0,
                                   cudaMemcpyDeviceToHost, st);
}
