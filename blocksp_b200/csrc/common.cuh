// common.cuh — shared device/host helpers for the BlockSp B200 kernels.
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include "../../include/blocksp_b200.h"

namespace bsp {

// Number of SMs on a B200; grids of persistent kernels are sized in multiples
// of the SM count read at handle creation, this is only the default.
constexpr int kB200SMs = 148;

// Bounded spin: a device-side wait on another warp's flag gives up after this
// many polls (each poll is followed by a short nanosleep), sets an error status
// and returns instead of hanging.  2^22 polls of >= 64 ns is well above any
// legitimate wait (a full triangular sweep takes well under a second).
constexpr unsigned kSpinLimit = 1u << 22;

// Device error word written by kernels: 0 = ok, else a bsp_status code.
struct DevStatus {
  int code;
  int where;  // row / item index that failed (diagnostic)
};

__device__ __forceinline__ void set_status(DevStatus* st, int code, int where) {
  if (st) {
    if (atomicCAS(&st->code, 0, code) == 0) st->where = where;
  }
}

// ---- 16-byte chunk of values: the unit every block stream is read in ----
template <typename VT> struct Chunk;
template <> struct Chunk<double> {
  using vec = double2;
  static constexpr int V = 2;
};
template <> struct Chunk<float> {
  using vec = float4;
  static constexpr int V = 4;
};
template <> struct Chunk<__nv_bfloat16> {
  using vec = uint4;
  static constexpr int V = 8;
};

// Streaming (evict-first) 16-byte load of matrix values: each block is read
// once per sweep, so it should not displace the vectors held in L2.
__device__ __forceinline__ double2 ld_stream(const double2* p) { return __ldcs(p); }
__device__ __forceinline__ float4 ld_stream(const float4* p) { return __ldcs(p); }
__device__ __forceinline__ uint4 ld_stream(const uint4* p) { return __ldcs(p); }

// Unpack a chunk into V accumulator-type values (FP32 or FP64 accumulation).
__device__ __forceinline__ void unpack(const double2& c, double* v) { v[0] = c.x; v[1] = c.y; }
template <typename AT> __device__ __forceinline__ void unpack(const float4& c, AT* v) {
  v[0] = c.x; v[1] = c.y; v[2] = c.z; v[3] = c.w;
}
template <typename AT> __device__ __forceinline__ void unpack(const uint4& c, AT* v) {
  const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&c);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    float2 f = __bfloat1622float2(h[i]);
    v[2 * i] = f.x;
    v[2 * i + 1] = f.y;
  }
}

// Load V consecutive accumulator-type vector entries (16-byte aligned).
// FP64 vectors next to FP64 (V = 2), FP32 (V = 4) or BF16 (V = 8) blocks.
template <int V> __device__ __forceinline__ void ld_vec(const double* p, double* v) {
  static_assert(V == 2 || V == 4 || V == 8, "chunks hold 2, 4 or 8 values");
#pragma unroll
  for (int k = 0; k < V / 2; ++k) {
    double2 t = __ldg(reinterpret_cast<const double2*>(p) + k);
    v[2 * k] = t.x;
    v[2 * k + 1] = t.y;
  }
}
template <int V> __device__ __forceinline__ void ld_vec(const float* p, float* v) {
  static_assert(V == 4 || V == 8, "float chunks hold 4 (fp32) or 8 (bf16) values");
  float4 t = __ldg(reinterpret_cast<const float4*>(p));
  v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
  if constexpr (V == 8) {
    float4 u = __ldg(reinterpret_cast<const float4*>(p) + 1);
    v[4] = u.x; v[5] = u.y; v[6] = u.z; v[7] = u.w;
  }
}
// Same, coherent at L2 (bypasses L1): used for vector entries written by other
// warps during the same launch (sync-free triangular sweeps).
template <int V> __device__ __forceinline__ void ld_vec_cg(const double* p, double* v) {
#pragma unroll
  for (int k = 0; k < V / 2; ++k) {
    double2 t = __ldcg(reinterpret_cast<const double2*>(p) + k);
    v[2 * k] = t.x;
    v[2 * k + 1] = t.y;
  }
}
template <int V> __device__ __forceinline__ void ld_vec_cg(const float* p, float* v) {
  float4 t = __ldcg(reinterpret_cast<const float4*>(p));
  v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
  if constexpr (V == 8) {
    float4 u = __ldcg(reinterpret_cast<const float4*>(p) + 1);
    v[4] = u.x; v[5] = u.y; v[6] = u.z; v[7] = u.w;
  }
}

// Acquire / release on a 32-bit flag at GPU scope.
__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// ---- the chunk map of one bs x bs block over a group of G lanes ----
// A block of BS*BS values of type VT is CPB = BS*BS/V 16-byte chunks laid out
// row-major, CPR = BS/V chunks per block row.  A group of G = min(32, CPB)
// lanes reads it in P = CPB/G passes; in pass p lane gl holds chunk p*G+gl,
// i.e. block row p*RPP + gl/CPR and columns (gl%CPR)*V .. +V-1.  Because G is
// a multiple of CPR the column offset of a lane is the same in every pass.
template <int BS, typename VT> struct BlockMap {
  static constexpr int V = Chunk<VT>::V;
  static_assert(BS % V == 0, "block row must be a whole number of 16-byte chunks");
  static constexpr int CPR = BS / V;
  static constexpr int CPB = BS * BS / V;
  static constexpr int G = CPB < 32 ? CPB : 32;
  static constexpr int P = CPB / G;
  static constexpr int RPP = G / CPR;
  static_assert(CPR <= 32 && (32 % G) == 0, "unsupported block size");
};

// Sum over the CPR lanes that share a block row (consecutive lanes).
template <int CPR, typename AT>
__device__ __forceinline__ AT row_reduce(AT v, unsigned mask) {
#pragma unroll
  for (int o = 1; o < CPR; o <<= 1) v += __shfl_xor_sync(mask, v, o);
  return v;
}

__host__ __device__ inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Process-wide count of kernel launches made by this library (bsp_launch_count).
void count_launch();
// Adds n (possibly negative) to the count: kernels replayed inside a CUDA graph.
void count_launch_add(int64_t n);

}  // namespace bsp

// ---- host-side error plumbing ----
#define BSP_CUDA_TRY(expr)                                                   \
  do {                                                                       \
    cudaError_t _e = (expr);                                                 \
    if (_e != cudaSuccess) {                                                 \
      bsp::record_error(std::string(#expr) + ": " + cudaGetErrorString(_e)); \
      return (_e == cudaErrorMemoryAllocation) ? BSP_OUT_OF_MEMORY           \
                                               : BSP_CUDA_ERROR;             \
    }                                                                        \
  } while (0)

#define BSP_TRY(expr)          \
  do {                         \
    int _s = (expr);           \
    if (_s != BSP_OK) return _s; \
  } while (0)

namespace bsp {
void record_error(const std::string& msg);
}
