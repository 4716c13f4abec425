// tma.cuh — Tensor Memory Accelerator (TMA) tile loads and mbarrier waits for the
// sm_100a stencil kernels.
//
// A field plane tile (with its halo) is fetched by one elected thread with
// cp.async.bulk.tensor.3d into shared memory; completion is tracked by an mbarrier
// transaction count.  Every wait is bounded in device time: after kWaitNs (%globaltimer)
// the waiting thread records an error in the kernel's error word and the kernel unwinds
// cleanly (the caller checks the word after the launch).  The limit is a time, not a
// poll count, because mbarrier.try_wait may suspend the thread for a hardware-defined
// interval on every call.  Tiles are never multicast.
//
// Alignment rules honoured by every caller: the innermost box coordinate x is a
// multiple of 4 floats (16 bytes), boxes are a multiple of 16 bytes wide, and the
// shared-memory destination of each box is 128-byte aligned.
#pragma once

#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

namespace gwmb {

constexpr unsigned long long kWaitNs = 1000000000ull;  // 1 s of device time before giving up

__device__ __forceinline__ unsigned long long device_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Deadline of one bounded wait: expired() turns true once kWaitNs have passed since its
// first call (the clock is read on the first call and then every 32nd).
struct WaitDeadline {
  unsigned long long t0 = 0;
  unsigned n = 0;
  __device__ __forceinline__ bool expired() {
    if (n++ == 0) {
      t0 = device_ns();
      return false;
    }
    return (n & 31u) == 0 && device_ns() - t0 > kWaitNs;
  }
};

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// make initialised barriers visible to the async (TMA) proxy
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// order earlier generic-proxy accesses of shared memory before later async-proxy writes
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for phase `parity` of an mbarrier.  Returns false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
  WaitDeadline d;
  while (!mbar_try_wait(bar, parity))
    if (d.expired()) return false;
  return true;
}

// 3-D tiled TMA load of box (x, y, z) of `map` into shared memory `dst`,
// completing on `bar`.  x must be a multiple of 4 (16 bytes of FP32).
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

}  // namespace gwmb
