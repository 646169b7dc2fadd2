// Bulk asynchronous copies global -> shared with mbarrier completion (sm_90+,
// used here on sm_100a): one thread issues a copy of a contiguous byte range,
// the copy engine moves it without registers, and the consumers wait on the
// stage's mbarrier.  No multicast anywhere: every source is this GPU's own
// memory, and each CTA fetches what it consumes.
//
// Every wait is bounded: a wait that has polled kWaitPolls times records
// kErrPipelineWait in the module's error word and returns false, and the
// kernel gives up its work (the host turns the word into VOX_ERR_TIMEOUT).
// Once the word is set, the other CTAs leave at their next check instead of
// waiting in turn.
#pragma once

#include <cstdint>

#include "vox_common.cuh"

namespace vox {

// Error word of the module (one per device): set by kernels that gave up a
// bounded wait, read and cleared by the host after each wait on a stream.
__device__ int g_kernel_err;
constexpr int kErrPipelineWait = 1;
constexpr unsigned kWaitPolls = 1u << 22;

// a wait elsewhere already gave up: kernels leave at once instead of waiting too
__device__ __forceinline__ bool kernel_err_set() {
  return *((volatile int*)&g_kernel_err) != 0;
}

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

// make the initialised barriers visible to the async (copy) proxy
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// true once the phase with the given parity has completed
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

// bounded wait; false (and the error word set) if the phase never completed
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
  for (unsigned i = 0; i < kWaitPolls; i++) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 1023u) == 1023u && kernel_err_set()) return false;
  }
  atomicOr(&g_kernel_err, kErrPipelineWait);
  return false;
}

// named barrier `id` over NT threads, true in all of them if pred is true in any
template <int NT>
__device__ __forceinline__ int named_bar_or(int id, int pred) {
  int r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.s32 p, %1, 0;\n\t"
      "bar.red.or.pred q, %2, %3, p;\n\t"
      "selp.s32 %0, 1, 0, q;\n\t}"
      : "=r"(r)
      : "r"(pred), "r"(id), "n"(NT)
      : "memory");
  return r;
}

// bytes (a multiple of 16, both addresses 16-byte aligned) from global src to
// shared dst, completing on bar's transaction count
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes,
                                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

}  // namespace vox
