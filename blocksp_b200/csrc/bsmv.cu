// bsmv.cu — block-sparse matrix x block vector on sm_100a.
//
// Replaces BlockSp::bsmv / mult_detail::blkSpMatVec (blocksp_multiply.hpp:166-325,
// 364-404): y = alpha * op(A) * x + beta * z for a BSR matrix with bs x bs
// row-major blocks and nrhs right-hand sides stored element-interleaved
// (the solArray<T,B,D> layout).
//
// Design: the blocks of one block row are contiguous in vals, so a group of G
// lanes streams them as 16-byte chunks (BlockMap): every load instruction of a
// warp reads 512 contiguous bytes, the blocks are read exactly once with
// evict-first caching, and x (which is re-read ~7 times for a 7-point stencil)
// stays resident in the 126 MB L2.  The CPR lanes that share a block row are
// reduced with shuffles.  This is an HBM-bound kernel: arithmetic intensity is
// 2 flop per stored value (R right-hand sides: 2R), far below any tensor-core
// ridge point, so it runs on the FP64/FP32 pipes.
#include "internal.hpp"

namespace bsp {

constexpr int kBsmvThreads = 256;
constexpr int kUnroll = 4;

template <int BS, typename VT, typename AT, int R>
__global__ void __launch_bounds__(kBsmvThreads)
k_bsmv(int n_rows, const int* __restrict__ row_ptr, const int* __restrict__ col_idx,
       const VT* __restrict__ vals, const AT* __restrict__ x, AT alpha, AT beta,
       const AT* z, AT* y) {
  using M = BlockMap<BS, VT>;
  using CV = typename Chunk<VT>::vec;
  constexpr int V = M::V, G = M::G, P = M::P, CPR = M::CPR, RPP = M::RPP, CPB = M::CPB;
  const int gl = threadIdx.x % G;
  const int row = blockIdx.x * (kBsmvThreads / G) + threadIdx.x / G;
  const bool valid = row < n_rows;
  const int c0 = (gl % CPR) * V;
  const CV* vblk = reinterpret_cast<const CV*>(vals);

  AT acc[P][R];
#pragma unroll
  for (int p = 0; p < P; ++p)
#pragma unroll
    for (int r = 0; r < R; ++r) acc[p][r] = AT(0);

  if (valid) {
    const int beg = __ldg(row_ptr + row), end = __ldg(row_ptr + row + 1);
    int j = beg;
    for (; j + kUnroll <= end; j += kUnroll) {
      int cols[kUnroll];
      CV a[kUnroll][P];
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) cols[u] = __ldg(col_idx + j + u);
#pragma unroll
      for (int u = 0; u < kUnroll; ++u)
#pragma unroll
        for (int p = 0; p < P; ++p)
          a[u][p] = ld_stream(vblk + (int64_t)(j + u) * CPB + p * G + gl);
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
          AT xv[V];
          ld_vec<V>(x + (int64_t)cols[u] * (BS * R) + r * BS + c0, xv);
#pragma unroll
          for (int p = 0; p < P; ++p) {
            AT av[V];
            unpack(a[u][p], av);
#pragma unroll
            for (int v = 0; v < V; ++v) acc[p][r] = fma(av[v], xv[v], acc[p][r]);
          }
        }
      }
    }
    for (; j < end; ++j) {
      const int col = __ldg(col_idx + j);
      CV a[P];
#pragma unroll
      for (int p = 0; p < P; ++p) a[p] = ld_stream(vblk + (int64_t)j * CPB + p * G + gl);
#pragma unroll
      for (int r = 0; r < R; ++r) {
        AT xv[V];
        ld_vec<V>(x + (int64_t)col * (BS * R) + r * BS + c0, xv);
#pragma unroll
        for (int p = 0; p < P; ++p) {
          AT av[V];
          unpack(a[p], av);
#pragma unroll
          for (int v = 0; v < V; ++v) acc[p][r] = fma(av[v], xv[v], acc[p][r]);
        }
      }
    }
  }
  // reduce the CPR lanes of each block row (all 32 lanes take part)
#pragma unroll
  for (int p = 0; p < P; ++p)
#pragma unroll
    for (int r = 0; r < R; ++r) acc[p][r] = row_reduce<CPR>(acc[p][r], 0xffffffffu);
  if (valid && (gl % CPR) == 0) {
#pragma unroll
    for (int p = 0; p < P; ++p)
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int64_t yi = (int64_t)row * (BS * R) + r * BS + p * RPP + gl / CPR;
        AT out = alpha * acc[p][r];
        if (beta != AT(0)) out += beta * z[yi];
        y[yi] = out;
      }
  }
}

// op(A) = A^T: gather over the block columns.  tr_ptr/tr_row/tr_blk list, for
// block column j, the blocks (row i, index t) of column j; the group owning
// output element j multiplies each block transposed (lane holds A[r][c0+v] and
// contributes A[r][c0+v] * x_i[r] to y_j[c0+v]).
template <int BS, typename VT, typename AT, int R>
__global__ void __launch_bounds__(kBsmvThreads)
k_bsmv_tr(int n_cols, const int* __restrict__ tr_ptr, const int* __restrict__ tr_row,
          const int64_t* __restrict__ tr_blk, const VT* __restrict__ vals,
          const AT* __restrict__ x, AT alpha, AT beta, const AT* z, AT* y) {
  using M = BlockMap<BS, VT>;
  using CV = typename Chunk<VT>::vec;
  constexpr int V = M::V, G = M::G, P = M::P, CPR = M::CPR, RPP = M::RPP, CPB = M::CPB;
  const int gl = threadIdx.x % G;
  const int colb = blockIdx.x * (kBsmvThreads / G) + threadIdx.x / G;
  const bool valid = colb < n_cols;
  const int c0 = (gl % CPR) * V;
  const CV* vblk = reinterpret_cast<const CV*>(vals);
  AT acc[R][V];
#pragma unroll
  for (int r = 0; r < R; ++r)
#pragma unroll
    for (int v = 0; v < V; ++v) acc[r][v] = AT(0);
  if (valid) {
    const int beg = __ldg(tr_ptr + colb), end = __ldg(tr_ptr + colb + 1);
    for (int t = beg; t < end; ++t) {
      const int i = __ldg(tr_row + t);
      const int64_t b = __ldg(tr_blk + t);
#pragma unroll
      for (int p = 0; p < P; ++p) {
        AT av[V];
        unpack(ld_stream(vblk + b * CPB + p * G + gl), av);
        const int rib = p * RPP + gl / CPR;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const AT xr = __ldg(x + (int64_t)i * (BS * R) + r * BS + rib);
#pragma unroll
          for (int v = 0; v < V; ++v) acc[r][v] = fma(av[v], xr, acc[r][v]);
        }
      }
    }
  }
  // lanes with equal gl % CPR hold partial sums of the same output entries
#pragma unroll
  for (int r = 0; r < R; ++r)
#pragma unroll
    for (int v = 0; v < V; ++v)
#pragma unroll
      for (int o = CPR; o < G; o <<= 1) acc[r][v] += __shfl_xor_sync(0xffffffffu, acc[r][v], o);
  if (valid && gl < CPR) {
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const int64_t yi = (int64_t)colb * (BS * R) + r * BS + c0 + v;
        AT out = alpha * acc[r][v];
        if (beta != AT(0)) out += beta * z[yi];
        y[yi] = out;
      }
  }
}

// Fallback for any block size / rhs count: one thread per output scalar.
template <typename VT, typename AT>
__global__ void k_bsmv_generic(int n_rows, int bs, int R, const int* __restrict__ row_ptr,
                               const int* __restrict__ col_idx, const VT* __restrict__ vals,
                               const AT* __restrict__ x, AT alpha, AT beta, const AT* z, AT* y) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t per_row = (int64_t)bs * R;
  if (idx >= (int64_t)n_rows * per_row) return;
  const int row = (int)(idx / per_row);
  const int rem = (int)(idx % per_row);
  const int r = rem / bs, t = rem % bs;
  AT acc = AT(0);
  for (int j = row_ptr[row]; j < row_ptr[row + 1]; ++j) {
    const int col = col_idx[j];
    const VT* a = vals + (int64_t)j * bs * bs + (int64_t)t * bs;
    const AT* xv = x + (int64_t)col * per_row + (int64_t)r * bs;
    for (int c = 0; c < bs; ++c) acc = fma(AT(a[c]), xv[c], acc);
  }
  AT out = alpha * acc;
  if (beta != AT(0)) out += beta * z[idx];
  y[idx] = out;
}

template <typename VT, typename AT>
__global__ void k_bsmv_tr_generic(int n_cols, int bs, int R, const int* __restrict__ tr_ptr,
                                  const int* __restrict__ tr_row, const int64_t* __restrict__ tr_blk,
                                  const VT* __restrict__ vals, const AT* __restrict__ x, AT alpha,
                                  AT beta, const AT* z, AT* y) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t per_row = (int64_t)bs * R;
  if (idx >= (int64_t)n_cols * per_row) return;
  const int colb = (int)(idx / per_row);
  const int rem = (int)(idx % per_row);
  const int r = rem / bs, c = rem % bs;
  AT acc = AT(0);
  for (int t = tr_ptr[colb]; t < tr_ptr[colb + 1]; ++t) {
    const int i = tr_row[t];
    const VT* a = vals + tr_blk[t] * bs * bs;
    const AT* xv = x + (int64_t)i * per_row + (int64_t)r * bs;
    for (int rr = 0; rr < bs; ++rr) acc = fma(AT(a[(int64_t)rr * bs + c]), xv[rr], acc);
  }
  AT out = alpha * acc;
  if (beta != AT(0)) out += beta * z[idx];
  y[idx] = out;
}

// ------------------------------------------------------------------------
template <int BS, typename VT, typename AT, int R>
static void launch_fwd(const bsp_matrix_s* A, const VT* vals, const AT* x, AT alpha, AT beta,
                       const AT* z, AT* y, cudaStream_t s) {
  constexpr int G = BlockMap<BS, VT>::G;
  const int rows_per_cta = kBsmvThreads / G;
  const int grid = (int)ceil_div(A->n_rows, rows_per_cta);
  bsp::count_launch(), k_bsmv<BS, VT, AT, R><<<grid, kBsmvThreads, 0, s>>>(A->n_rows, A->row_ptr.get(),
                                                      A->col_idx.get(), vals, x, alpha, beta, z, y);
}
template <int BS, typename VT, typename AT, int R>
static void launch_tr(const bsp_matrix_s* A, const VT* vals, const AT* x, AT alpha, AT beta,
                      const AT* z, AT* y, cudaStream_t s) {
  constexpr int G = BlockMap<BS, VT>::G;
  const int per_cta = kBsmvThreads / G;
  const int grid = (int)ceil_div(A->n_cols, per_cta);
  bsp::count_launch(), k_bsmv_tr<BS, VT, AT, R><<<grid, kBsmvThreads, 0, s>>>(
      A->n_cols, A->tr_ptr.get(), A->tr_row.get(), A->tr_blk.get(), vals, x, alpha, beta, z, y);
}

template <int BS, typename VT, typename AT>
static bool dispatch_r(const bsp_matrix_s* A, int R, bool tr, const VT* vals, const AT* x,
                       AT alpha, AT beta, const AT* z, AT* y, cudaStream_t s) {
  if constexpr (BS % Chunk<VT>::V != 0) {
    return false;
  } else {
    switch (R) {
#define BSP_R_CASE(RR)                                                  \
  case RR:                                                              \
    if (tr) launch_tr<BS, VT, AT, RR>(A, vals, x, alpha, beta, z, y, s); \
    else launch_fwd<BS, VT, AT, RR>(A, vals, x, alpha, beta, z, y, s);   \
    return true;
      BSP_R_CASE(1)
      BSP_R_CASE(2)
      BSP_R_CASE(3)
      BSP_R_CASE(4)
#undef BSP_R_CASE
      default:
        return false;
    }
  }
}

template <typename VT, typename AT>
static int bsmv_typed(const bsp_matrix_s* A, int R, bool tr, const VT* vals, const AT* x,
                      AT alpha, AT beta, const AT* z, AT* y, cudaStream_t s) {
  bool done = false;
  switch (A->bs) {
    case 2: done = dispatch_r<2, VT, AT>(A, R, tr, vals, x, alpha, beta, z, y, s); break;
    case 4: done = dispatch_r<4, VT, AT>(A, R, tr, vals, x, alpha, beta, z, y, s); break;
    case 8: done = dispatch_r<8, VT, AT>(A, R, tr, vals, x, alpha, beta, z, y, s); break;
    case 16: done = dispatch_r<16, VT, AT>(A, R, tr, vals, x, alpha, beta, z, y, s); break;
    case 32: done = dispatch_r<32, VT, AT>(A, R, tr, vals, x, alpha, beta, z, y, s); break;
    default: break;
  }
  if (!done) {
    const int64_t total = (int64_t)(tr ? A->n_cols : A->n_rows) * A->bs * R;
    const int threads = 256;
    const int64_t grid = ceil_div(total, threads);
    if (grid > 0) {
      if (tr)
        bsp::count_launch(), k_bsmv_tr_generic<VT, AT><<<(unsigned)grid, threads, 0, s>>>(
            A->n_cols, A->bs, R, A->tr_ptr.get(), A->tr_row.get(), A->tr_blk.get(), vals, x,
            alpha, beta, z, y);
      else
        bsp::count_launch(), k_bsmv_generic<VT, AT><<<(unsigned)grid, threads, 0, s>>>(
            A->n_rows, A->bs, R, A->row_ptr.get(), A->col_idx.get(), vals, x, alpha, beta, z, y);
    }
  }
  BSP_CUDA_TRY(cudaPeekAtLastError());
  return BSP_OK;
}

int build_transpose(bsp_matrix_s* A);

// Entry used by the C ABI and by the solvers.
int bsmv_launch(bsp_matrix_s* A, int nrhs, int transpose, int dtype, double alpha,
                const void* x, double beta, const void* z, void* y, cudaStream_t s) {
  if (nrhs < 1) return BSP_INVALID;
  if (transpose && !A->has_transpose) BSP_TRY(build_transpose(A));
  const bool tr = transpose != 0;
  if (A->n_rows == 0 || A->n_cols == 0) return BSP_OK;
  switch (dtype) {
    case BSP_F64:
      return bsmv_typed<double, double>(A, nrhs, tr, A->vals.get(), (const double*)x, alpha,
                                        beta, (const double*)z, (double*)y, s);
    case BSP_F32:
      if (!A->vals32.get()) return BSP_INVALID;
      return bsmv_typed<float, float>(A, nrhs, tr, A->vals32.get(), (const float*)x, (float)alpha,
                                      (float)beta, (const float*)z, (float*)y, s);
    case BSP_BF16:
      if (!A->vals16.get()) return BSP_INVALID;
      return bsmv_typed<__nv_bfloat16, float>(A, nrhs, tr, A->vals16.get(), (const float*)x,
                                              (float)alpha, (float)beta, (const float*)z,
                                              (float*)y, s);
    case BSP_F32_STORE:  // FP32 blocks, FP64 vectors and accumulation
      if (!A->vals32.get()) return BSP_INVALID;
      return bsmv_typed<float, double>(A, nrhs, tr, A->vals32.get(), (const double*)x, alpha, beta,
                                       (const double*)z, (double*)y, s);
    case BSP_BF16_STORE:  // BF16 blocks, FP64 vectors and accumulation
      if (!A->vals16.get()) return BSP_INVALID;
      return bsmv_typed<__nv_bfloat16, double>(A, nrhs, tr, A->vals16.get(), (const double*)x, alpha,
                                               beta, (const double*)z, (double*)y, s);
    default:
      return BSP_INVALID;
  }
}

// Build the block-column index of A on the host from its structure.
int build_transpose(bsp_matrix_s* A) {
  const int nc = A->n_cols;
  std::vector<int> ptr(nc + 1, 0);
  for (int64_t t = 0; t < A->nnzb; ++t) ptr[A->h_col_idx[t] + 1]++;
  for (int j = 0; j < nc; ++j) ptr[j + 1] += ptr[j];
  std::vector<int> rows(A->nnzb);
  std::vector<int64_t> blk(A->nnzb);
  std::vector<int> fill(ptr.begin(), ptr.end() - 1);
  // rows visited in increasing order, so every column lists its rows sorted:
  // the accumulation order of the reference's transpose path over getIndices()
  // (blocksp_containers.hpp:380-387, blocksp_multiply.hpp:280-284).
  for (int i = 0; i < A->n_rows; ++i)
    for (int t = A->h_row_ptr[i]; t < A->h_row_ptr[i + 1]; ++t) {
      const int j = A->h_col_idx[t];
      rows[fill[j]] = i;
      blk[fill[j]] = t;
      fill[j]++;
    }
  BSP_TRY(A->tr_ptr.alloc(nc + 1));
  BSP_TRY(A->tr_row.alloc(A->nnzb > 0 ? A->nnzb : 1));
  BSP_TRY(A->tr_blk.alloc(A->nnzb > 0 ? A->nnzb : 1));
  BSP_CUDA_TRY(cudaMemcpy(A->tr_ptr.get(), ptr.data(), (nc + 1) * sizeof(int), cudaMemcpyHostToDevice));
  if (A->nnzb > 0) {
    BSP_CUDA_TRY(cudaMemcpy(A->tr_row.get(), rows.data(), A->nnzb * sizeof(int), cudaMemcpyHostToDevice));
    BSP_CUDA_TRY(cudaMemcpy(A->tr_blk.get(), blk.data(), A->nnzb * sizeof(int64_t), cudaMemcpyHostToDevice));
  }
  A->has_transpose = true;
  return BSP_OK;
}

}  // namespace bsp
