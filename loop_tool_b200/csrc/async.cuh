// mbarrier and bulk-copy helpers shared by the kernels that stage global
// memory through shared memory with the TMA engine (inline PTX, sm_100a).
// Every wait is bounded: after kWaitCycles (about 2 s) or once another CTA
// has raised the flag, the wait sets *err and reports failure so the caller
// can wind down instead of hanging the GPU.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace {

constexpr long long kWaitCycles = 4000000000LL;  // ~2 s at 1.9 GHz
// The error flag lives in global memory: a wait reads it only once it has
// lasted this long (~50 us), so ordinary hand-offs never pay a global load's
// latency between two polls of the barrier.
constexpr long long kFlagCycles = 100000LL;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n"
      " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Wait at most `limit` cycles for the phase of parity `parity` to complete
// (giving up early once another CTA has raised *err); on giving up, raise
// *err and return false.
__device__ __forceinline__ bool mbar_wait_for(uint32_t bar, uint32_t parity, int* err,
                                              long long limit) {
  if (mbar_try(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try(bar, parity)) {
    const long long dt = clock64() - t0;
    if (dt > limit || (dt > kFlagCycles && *(volatile int*)err)) {
      atomicExch(err, 1);
      return false;
    }
  }
  return true;
}

// Bounded wait for the phase of parity `parity` to complete.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int* err) {
  return mbar_wait_for(bar, parity, err, kWaitCycles);
}

// Bounded wait that ignores the error flag: used while winding down, to let
// copies already in flight land before the CTA exits.
__device__ __forceinline__ bool mbar_drain(uint32_t bar, uint32_t parity) {
  const long long t0 = clock64();
  while (!mbar_try(bar, parity))
    if (clock64() - t0 > kWaitCycles) return false;
  return true;
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}

// 1-D bulk copy global -> shared (TMA, no tensor map) completing on an
// mbarrier's transaction count.  dst / src 16-byte aligned, bytes a
// multiple of 16.
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes,
                                          uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      ::"r"(dst), "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

}  // namespace
