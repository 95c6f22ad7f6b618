// sentinel.cuh — publication of sweep results by their values.
#pragma once
#include "common.cuh"

namespace bsp {

// A sweep's output vector is filled with a signalling-NaN bit pattern before
// the launch.  Arithmetic never produces it (NaN results are quiet), so a row
// is final exactly when its words differ from the pattern.  Aligned 8- and
// 4-byte accesses are single-copy atomic, so a reader never sees half a value.
constexpr unsigned long long kSentinel64 = 0x7FF4B5B5B5B5B5B5ull;
constexpr unsigned kSentinel32 = 0x7FA5B5B5u;
__device__ __forceinline__ bool is_sentinel(double v) {
  return (unsigned long long)__double_as_longlong(v) == kSentinel64;
}
__device__ __forceinline__ bool is_sentinel(float v) { return __float_as_uint(v) == kSentinel32; }
// Re-reads inside a polling loop: relaxed loads at GPU scope, never merged.
__device__ __forceinline__ double ld_poll(const double* p) {
  double v;
  asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ float ld_poll(const float* p) {
  float v;
  asm volatile("ld.relaxed.gpu.global.f32 %0, [%1];" : "=f"(v) : "l"(p) : "memory");
  return v;
}

// Pause between polls of a value another group is about to publish: the first
// polls re-read at once (the producer is usually a few hundred cycles away),
// later ones back off so long waits do not flood L2 with re-reads.
constexpr unsigned kSpinFree = 32;
__device__ __forceinline__ void poll_pause(unsigned spins) {
  if (spins >= kSpinFree) __nanosleep(spins >= 1024 ? 256 : 32);
}

}  // namespace bsp
