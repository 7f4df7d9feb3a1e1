// psg_tma.cuh -- bulk asynchronous copies (TMA, cp.async.bulk) and mbarrier
// helpers for sm_100a, written as inline PTX.
//
// A tile that is one contiguous chunk of global memory is moved into shared
// memory by a single cp.async.bulk issued by one thread; completion is tracked
// by an mbarrier transaction count.  Waits are bounded: when a wait runs out
// the kernel records PSG_DEV_TIMEOUT in its status word and the caller returns.
#pragma once
#include <stdint.h>

#include "psg_common.cuh"

#define PSG_DEV_TIMEOUT 0x7e01

namespace psg {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// dst (shared), src (global): 16-byte aligned; bytes: a multiple of 16
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// prefetch a contiguous chunk (16-byte aligned, size a multiple of 16) into L2
__device__ __forceinline__ void bulk_prefetch_l2(const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Wait for phase `parity` of `bar`, at most ~2^22 polls (each poll suspends
// for a hardware-bounded time).  Returns false after recording a timeout.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int* status) {
  for (int i = 0; i < (1 << 22); ++i)
    if (mbar_try_wait(bar, parity)) return true;
  if (status) atomicExch(status, PSG_DEV_TIMEOUT);
  return false;
}

// the same with a caller-chosen number of polls
__device__ __forceinline__ bool mbar_wait_polls(uint64_t* bar, uint32_t parity, int polls,
                                                int* status) {
  for (int i = 0; i < polls; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  if (status) atomicExch(status, PSG_DEV_TIMEOUT);
  return false;
}

// Block-wide load of `nchunks` contiguous chunks into shared memory through one
// mbarrier: thread 0 arms the barrier and issues the copies, every thread waits.
// Returns false (uniformly) when the wait timed out.
struct BulkLoad {
  uint64_t* bar;
  uint32_t phase;
};

}  // namespace psg
