// blockops.cuh — warp-level dense operations on one bs x bs block (bs <= 32).
//
// Used by the preconditioner set-up kernels (block ILU0 / IChol0 factorisation
// and diagonal-block inversion).  A warp owns one block row at a time; the
// blocks it works on are staged in the warp's slice of shared memory,
// row-major, and every routine ends with __syncwarp() so the result is visible
// to all 32 lanes.
#pragma once
#include "common.cuh"

namespace bsp {

__device__ __forceinline__ void warp_copy_in(double* s, const double* g, int nel) {
  const int lane = threadIdx.x & 31;
  for (int e = lane; e < nel; e += 32) s[e] = __ldcg(g + e);
  __syncwarp();
}
__device__ __forceinline__ void warp_copy_out(double* g, const double* s, int nel) {
  const int lane = threadIdx.x & 31;
  for (int e = lane; e < nel; e += 32) g[e] = s[e];
  __syncwarp();
}

// The routines below take the block size as a template argument BS when it
// is known at compile time (loops unrolled, index arithmetic by shifts) and
// at run time otherwise (BS = 0); both forms do the same operations in the
// same order.

// C = A * B (trB = 0) or C = A * B^T (trB = 1); C must not alias A or B.
template <int BS = 0>
__device__ inline void warp_gemm(double* C, const double* A, const double* B, int bs_rt, bool trB) {
  const int bs = BS > 0 ? BS : bs_rt;
  const int lane = threadIdx.x & 31;
  for (int e = lane; e < bs * bs; e += 32) {
    const int r = e / bs, c = e % bs;
    double acc = 0.0;
    if (trB) {
#pragma unroll
      for (int t = 0; t < (BS > 0 ? BS : bs); ++t) acc = fma(A[r * bs + t], B[c * bs + t], acc);
    } else {
#pragma unroll
      for (int t = 0; t < (BS > 0 ? BS : bs); ++t) acc = fma(A[r * bs + t], B[t * bs + c], acc);
    }
    C[e] = acc;
  }
  __syncwarp();
}

// G -= A * B (trB = 0) or G -= A * B^T; G is a global block owned by this warp.
__device__ inline void warp_gemm_sub_global(double* G, const double* A, const double* B, int bs,
                                            bool trB) {
  const int lane = threadIdx.x & 31;
  for (int e = lane; e < bs * bs; e += 32) {
    const int r = e / bs, c = e % bs;
    double acc = 0.0;
    if (trB)
      for (int t = 0; t < bs; ++t) acc = fma(A[r * bs + t], B[c * bs + t], acc);
    else
      for (int t = 0; t < bs; ++t) acc = fma(A[r * bs + t], B[t * bs + c], acc);
    G[e] = __ldcg(G + e) - acc;
  }
  __syncwarp();
}

// Gauss-Jordan inverse with the augmented matrix [M | I] held by columns in
// registers: lane c (c < 2 BS) keeps column c.  The same pivots, divisions
// and FMAs as the shared-memory form below, without its shared-memory round
// trips and warp barriers per step.
template <int BS>
__device__ inline bool warp_inverse_cols(double* Inv, const double* M) {
  const int lane = threadIdx.x & 31;
  constexpr int W2 = 2 * BS;
  double col[BS];
#pragma unroll
  for (int r = 0; r < BS; ++r)
    col[r] = lane < BS ? M[r * BS + lane] : (lane < W2 && lane - BS == r ? 1.0 : 0.0);
  bool ok = true;
#pragma unroll
  for (int k = 0; k < BS; ++k) {
    // pivot: the largest |aug[r][k]| over r >= k, the lowest row on ties, a
    // NaN never chosen over a number (lane k scans its column)
    double best = -1.0;
    int bidx = k;
#pragma unroll
    for (int r = k; r < BS; ++r) {
      double v = fabs(col[r]);
      if (v != v) v = -0.5;
      if (v > best) {
        best = v;
        bidx = r;
      }
    }
    best = __shfl_sync(0xffffffffu, best, k);
    bidx = __shfl_sync(0xffffffffu, bidx, k);
    if (!(best > 0.0) || !isfinite(best)) ok = false;
    if (bidx != k) {  // rows k and bidx swap in every column
      double tb = 0.0;
#pragma unroll
      for (int r = k + 1; r < BS; ++r)
        if (r == bidx) tb = col[r];
#pragma unroll
      for (int r = k + 1; r < BS; ++r)
        if (r == bidx) col[r] = col[k];
      col[k] = tb;
    }
    const double piv = __shfl_sync(0xffffffffu, col[k], k);
    col[k] = col[k] / piv;
    // eliminate column k from the other rows with the multipliers aug[r][k]
#pragma unroll
    for (int r = 0; r < BS; ++r) {
      if (r == k) continue;
      const double mult = __shfl_sync(0xffffffffu, col[r], k);
      if (lane != k) col[r] = fma(-mult, col[k], col[r]);
    }
    if (lane == k) {
#pragma unroll
      for (int r = 0; r < BS; ++r)
        if (r != k) col[r] = 0.0;
    }
  }
  if (lane >= BS && lane < W2) {
#pragma unroll
    for (int r = 0; r < BS; ++r) Inv[r * BS + (lane - BS)] = col[r];
  }
  __syncwarp();
  return ok;
}

// Inverse by Gauss-Jordan elimination with partial (row) pivoting.
// M (bs x bs) is destroyed; aug is scratch of bs*2*bs doubles.  Returns false
// when a pivot is exactly zero or not finite (singular block).
template <int BS = 0>
__device__ inline bool warp_inverse(double* Inv, const double* M, double* aug, int bs_rt) {
  if constexpr (BS > 0 && BS <= 16) return warp_inverse_cols<BS>(Inv, M);
  const int bs = BS > 0 ? BS : bs_rt;
  const int lane = threadIdx.x & 31;
  const int w = 2 * bs;
  for (int e = lane; e < bs * w; e += 32) {
    const int r = e / w, c = e % w;
    aug[e] = c < bs ? M[r * bs + c] : (c - bs == r ? 1.0 : 0.0);
  }
  __syncwarp();
  bool ok = true;
  for (int k = 0; k < bs; ++k) {
    // pivot search over rows k..bs-1 (lane r holds row r)
    double best = -1.0;
    int bidx = k;
    if (lane >= k && lane < bs) {
      best = fabs(aug[lane * w + k]);
      if (best != best) best = -0.5;  // NaN never wins the comparison below
      bidx = lane;
    }
    // the candidates sit in lanes 0..bs-1: a butterfly over the smallest
    // power-of-two segment that holds them (the whole warp when bs is known
    // only at run time)
    constexpr int SEG = BS <= 0 ? 32 : BS <= 4 ? 4 : BS <= 8 ? 8 : BS <= 16 ? 16 : 32;
#pragma unroll
    for (int o = SEG / 2; o > 0; o >>= 1) {
      const double ob = __shfl_xor_sync(0xffffffffu, best, o, SEG);
      const int oi = __shfl_xor_sync(0xffffffffu, bidx, o, SEG);
      if (ob > best || (ob == best && oi < bidx)) { best = ob; bidx = oi; }
    }
    // Every lane must take the same pivot: the row swap below is a branch that
    // contains __syncwarp().  Broadcast lane 0's choice so the control flow is
    // warp-uniform whatever the values (NaN or Inf from a failed block).
    best = __shfl_sync(0xffffffffu, best, 0);
    bidx = __shfl_sync(0xffffffffu, bidx, 0);
    if (!(best > 0.0) || !isfinite(best)) ok = false;
    if (bidx != k) {
      for (int c = lane; c < w; c += 32) {
        const double t = aug[k * w + c];
        aug[k * w + c] = aug[bidx * w + c];
        aug[bidx * w + c] = t;
      }
      __syncwarp();
    }
    const double piv = aug[k * w + k];
    __syncwarp();
    for (int c = lane; c < w; c += 32) aug[k * w + c] = aug[k * w + c] / piv;
    __syncwarp();
    // eliminate column k from every other row; column k itself is left
    // untouched during the update (it holds the multipliers) and zeroed after
    for (int e = lane; e < bs * w; e += 32) {
      const int r = e / w, c = e % w;
      if (r == k || c == k) continue;
      aug[e] = fma(-aug[r * w + k], aug[k * w + c], aug[e]);
    }
    __syncwarp();
    for (int r = lane; r < bs; r += 32)
      if (r != k) aug[r * w + k] = 0.0;
    __syncwarp();
  }
  for (int e = lane; e < bs * bs; e += 32) {
    const int r = e / bs, c = e % bs;
    Inv[e] = aug[r * w + bs + c];
  }
  __syncwarp();
  return ok;
}

// In-place lower Cholesky A = L L^T (upper triangle zeroed), row-oriented
// (Cholesky-Banachiewicz).  Returns false on a non-positive pivot.
template <int BS = 0>
__device__ inline bool warp_cholesky(double* A, int bs_rt) {
  const int bs = BS > 0 ? BS : bs_rt;
  const int lane = threadIdx.x & 31;
  bool ok = true;
  for (int j = 0; j < bs; ++j) {
    // diagonal: A[j][j] - sum_{t<j} L[j][t]^2
    double part = 0.0;
    for (int t = lane; t < j; t += 32) part = fma(A[j * bs + t], A[j * bs + t], part);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
    const double d = A[j * bs + j] - part;
    if (!(d > 0.0) || !isfinite(d)) ok = false;
    const double ljj = sqrt(d);
    __syncwarp();
    // column below the diagonal: lane r computes L[r][j]
    for (int r = j + 1 + lane; r < bs; r += 32) {
      double acc = 0.0;
      for (int t = 0; t < j; ++t) acc = fma(A[r * bs + t], A[j * bs + t], acc);
      A[r * bs + j] = (A[r * bs + j] - acc) / ljj;
    }
    __syncwarp();
    if (lane == 0) A[j * bs + j] = ljj;
    __syncwarp();
  }
  for (int e = lane; e < bs * bs; e += 32)
    if (e % bs > e / bs) A[e] = 0.0;
  __syncwarp();
  return ok;
}

// Inverse of a lower-triangular L (bs <= 32): lane c solves column c.
template <int BS = 0>
__device__ inline void warp_lower_inverse(double* X, const double* L, int bs_rt) {
  const int bs = BS > 0 ? BS : bs_rt;
  const int lane = threadIdx.x & 31;
  if (lane < bs) {
    const int c = lane;
    for (int r = 0; r < bs; ++r) {
      double acc = (r == c) ? 1.0 : 0.0;
      for (int t = c; t < r; ++t) acc = fma(-L[r * bs + t], X[t * bs + c], acc);
      X[r * bs + c] = (r < c) ? 0.0 : acc / L[r * bs + r];
    }
  }
  __syncwarp();
}

// Find column `key` in the sorted list cols[beg, end); returns its index or -1.
__device__ inline int warp_find(const int* __restrict__ cols, int beg, int end, int key) {
  const int lane = threadIdx.x & 31;
  for (int base = beg; base < end; base += 32) {
    const int e = base + lane;
    const bool hit = e < end && __ldg(cols + e) == key;
    const unsigned m = __ballot_sync(0xffffffffu, hit);
    if (m) return base + __ffs(m) - 1;
  }
  return -1;
}

}  // namespace bsp
