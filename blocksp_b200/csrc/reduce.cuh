// reduce.cuh — deterministic fused grid reductions.
//
// A reduction launch has a fixed grid (kRedBlocks CTAs), a grid-stride body
// that may also write vectors (fused axpy + dot), a fixed-shape block tree,
// and a "last CTA" epilogue that sums the per-CTA partials in index order and
// runs a finaliser on one thread.  The result therefore does not depend on
// scheduling: the same inputs give bit-identical scalars on every run, which
// is what lets solver histories be compared against the CPU oracle.
#pragma once
#include "internal.hpp"

namespace bsp {

constexpr int kRedThreads = 512;

template <int NV>
__device__ __forceinline__ void block_reduce_store(double (&v)[NV], double* out) {
  __shared__ double sm[NV][kRedThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double t = v[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (lane == 0) sm[k][warp] = t;
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double t = lane < (kRedThreads / 32) ? sm[k][lane] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
      if (lane == 0) out[k] = t;
    }
  }
}

// Body: __device__ void setup() once per thread (loads device scalars), then
//       __device__ void operator()(int64_t i, double (&acc)[NV]) for element i.
// Fin:  __device__ void operator()(const double (&sum)[NV]) on one thread.
template <int NV, class Body, class Fin>
__global__ void __launch_bounds__(kRedThreads)
k_reduce(int64_t n, Body body, Fin fin, double* partials, unsigned* ticket) {
  double acc[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k) acc[k] = 0.0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  Body b = body;
  b.setup();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) b(i, acc);
  __shared__ double blk[NV];
  block_reduce_store<NV>(acc, blk);
  __shared__ bool last;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) partials[blockIdx.x * NV + k] = blk[k];
    __threadfence();
    last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double s[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k) s[k] = 0.0;
  for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x)
#pragma unroll
    for (int k = 0; k < NV; ++k) s[k] += __ldcg(partials + b * NV + k);
  __shared__ double tot[NV];
  __syncthreads();
  block_reduce_store<NV>(s, tot);
  __syncthreads();
  if (threadIdx.x == 0) {
    fin(tot);
    *ticket = 0u;  // ready for the next launch on this slot
  }
}

// Launch on reduction slot `slot` of the handle's workspace.
template <int NV, class Body, class Fin>
inline int launch_reduce(bsp_handle_s* h, int slot, int64_t n, Body body, Fin fin) {
  double* partials = h->ws.partials.get() + (size_t)slot * kRedBlocks * 4;
  unsigned* ticket = h->ws.tickets.get() + slot;
  static_assert(NV <= 4, "at most 4 simultaneous sums per launch");
  bsp::count_launch(), k_reduce<NV, Body, Fin><<<kRedBlocks, kRedThreads, 0, h->stream>>>(n, body, fin, partials, ticket);
  BSP_CUDA_TRY(cudaPeekAtLastError());
  return BSP_OK;
}

// ---- common bodies / finalisers ----
struct DotBody {
  const double* x;
  const double* y;
  __device__ void setup() {}
  __device__ void operator()(int64_t i, double (&a)[1]) const { a[0] = fma(x[i], y[i], a[0]); }
};
struct StoreFin {
  double* out;
  __device__ void operator()(const double (&s)[1]) const { *out = s[0]; }
};

}  // namespace bsp
