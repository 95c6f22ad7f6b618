// stage.cuh — per-thread asynchronous staging of global data in shared memory.
//
// cp.async copies global memory to shared memory without holding registers;
// a thread groups its copies (commit_group) and later waits until at most N
// of its most recent groups are still in flight (wait_group N).  Each thread
// copies the bytes it will read itself, so completion needs no barrier.
// Both addresses must be aligned to the copy size (4, 8 or 16 bytes).
#pragma once
#include <cstdint>
#include "common.cuh"

namespace bsp {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// 16 bytes, cached in L2 only (streamed matrix blocks).
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}

// 4, 8 or 16 bytes (vector values).
template <int N> __device__ __forceinline__ void cp_async_small(void* dst, const void* src) {
  static_assert(N == 4 || N == 8 || N == 16, "cp.async copies 4, 8 or 16 bytes");
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(smem_addr(dst)), "l"(src), "n"(N) : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }

// Waits until at most N of this thread's most recent groups are pending.
template <int N> __device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

}  // namespace bsp
