// bsmm.cu — block sparse identity, transpose, sum and matrix-matrix product.
//
// Reference: blocksp_multiply.hpp:21-45 (blkSpIdent, blkSpTranspose),
// :51-133 (blkSpMatMat, C = A B and C = A^T B), :137-159 (triple and
// quadruple products, right-nested), :335-362 (bs_id, bs_tr, bsmm) and
// blocksp_containers.hpp:302-318, :340-347 (+=, -=, *= of the CSR container).
//
// The structure of every result is built on the host from the matrices' host
// structure copies, in the order the reference's container creates blocks:
// BlockSp's operator() appends a missing block at the end of its row, so a
// row of C lists its blocks in order of first creation by the reference's
// loops.  The values are computed on the GPU:
//   * product: one warp per block of C; the contributing block pairs are
//     listed per C block in the reference's order of addition, each pair's
//     product P = A_ik B_kj is formed with the inner index ascending (as
//     dense::matMat's loops do) and added to C_ij in that order;
//   * A^T B: the reference forms A_ik^T B_ij with the same inner order; here
//     A^T is built first (bs_tr) and the plain product runs on it, which is
//     the same sequence of operations;
//   * transpose, identity and alpha A + beta B are gathers.
#include <algorithm>
#include <vector>
#include "internal.hpp"

namespace bsp {

int grid_for(const bsp_handle_s* h, int64_t n, int threads);

constexpr int kMMWarps = 4;

// C[c] = sum over pairs t of C block c (pair_ptr) of A[pa[t]] * B[pb[t]]
__global__ void __launch_bounds__(kMMWarps * 32)
    k_bsmm(int64_t n_cblk, int bs, const int64_t* __restrict__ pair_ptr, const int* __restrict__ pa,
           const int* __restrict__ pb, const double* __restrict__ A, const double* __restrict__ B,
           double* __restrict__ C) {
  extern __shared__ double mm_smem[];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int b2 = bs * bs;
  double* sa = mm_smem + (size_t)w * 2 * b2;
  double* sb = sa + b2;
  for (int64_t c = (int64_t)blockIdx.x * kMMWarps + w; c < n_cblk; c += (int64_t)gridDim.x * kMMWarps) {
    double acc[32];
    const int nout = (b2 + 31) / 32;
#pragma unroll
    for (int u = 0; u < 32; ++u) acc[u] = 0.0;
    for (int64_t t = pair_ptr[c]; t < pair_ptr[c + 1]; ++t) {
      const double* a = A + (int64_t)pa[t] * b2;
      const double* b = B + (int64_t)pb[t] * b2;
      for (int e = lane; e < b2; e += 32) {
        sa[e] = a[e];
        sb[e] = b[e];
      }
      __syncwarp();
#pragma unroll
      for (int u = 0; u < 32; ++u) {
        if (u >= nout) break;
        const int e = lane + 32 * u;
        if (e < b2) {
          const int r = e / bs, col = e - r * bs;
          double p = 0.0;
          for (int k = 0; k < bs; ++k) p = fma(sa[r * bs + k], sb[k * bs + col], p);
          acc[u] += p;
        }
      }
      __syncwarp();
    }
#pragma unroll
    for (int u = 0; u < 32; ++u) {
      if (u >= nout) break;
      const int e = lane + 32 * u;
      if (e < b2) C[c * b2 + e] = acc[u];
    }
  }
}

// dst[e] = alpha * (ia[e] >= 0 ? A[ia[e]] : 0) + beta * (ib[e] >= 0 ? B[ib[e]] : 0), per block,
// transposed when trans (then only ia is used).
__global__ void k_block_combine(int64_t nblk, int bs, const int64_t* __restrict__ ia, const int64_t* __restrict__ ib,
                                const double* __restrict__ A, const double* __restrict__ B, double alpha,
                                double beta, int trans, double* __restrict__ dst) {
  const int b2 = bs * bs;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nblk * b2;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = t / b2;
    const int k = (int)(t - e * b2);
    const int r = k / bs, c = k - r * bs;
    const int ks = trans ? c * bs + r : k;
    const int64_t a = ia ? ia[e] : -1, b = ib ? ib[e] : -1;
    double v;
    if (a >= 0 && b >= 0) v = alpha * A[a * b2 + ks] + beta * B[b * b2 + ks];
    else if (a >= 0) v = alpha == 1.0 ? A[a * b2 + ks] : alpha * A[a * b2 + ks];
    else v = beta == 1.0 ? B[b * b2 + ks] : beta * B[b * b2 + ks];
    dst[t] = v;
  }
}

__global__ void k_identity_blocks(int64_t n, int bs, double* __restrict__ dst) {
  const int b2 = bs * bs;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n * b2; t += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(t % b2);
    dst[t] = (k / bs == k % bs) ? 1.0 : 0.0;
  }
}

template <typename T> static int upload_tmp(DevBuf<T>& d, const std::vector<T>& v) {
  BSP_TRY(d.alloc(std::max<size_t>(v.size(), 1)));
  if (!v.empty()) BSP_CUDA_TRY(cudaMemcpy(d.get(), v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  return BSP_OK;
}

// Host structure of the block transpose: row j lists (i, block of A_ij) for
// increasing i, i.e. the order blkSpTranspose's loops create them.
static void transpose_struct(const bsp_matrix_s* A, std::vector<int>& ptr, std::vector<int>& col,
                             std::vector<int64_t>& src) {
  const int m = A->n_rows, n = A->n_cols;
  ptr.assign(n + 1, 0);
  for (int64_t t = 0; t < A->nnzb; ++t) ptr[A->h_col_idx[t] + 1]++;
  for (int j = 0; j < n; ++j) ptr[j + 1] += ptr[j];
  col.resize(A->nnzb);
  src.resize(A->nnzb);
  std::vector<int> fill(ptr.begin(), ptr.end() - 1);
  for (int i = 0; i < m; ++i)
    for (int t = A->h_row_ptr[i]; t < A->h_row_ptr[i + 1]; ++t) {
      const int j = A->h_col_idx[t];
      col[fill[j]] = i;
      src[fill[j]] = t;
      fill[j]++;
    }
}

static int make_matrix(bsp_handle_t h, int m, int n, int bs, const std::vector<int>& ptr, const std::vector<int>& col,
                       bsp_matrix_t* out) {
  return matrix_create_struct(h, m, n, bs, (int64_t)col.size(), ptr.data(), col.empty() ? nullptr : col.data(),
                              out);
}

}  // namespace bsp

using namespace bsp;

extern "C" {

int bsp_bs_id(bsp_handle_t h, int n, int bs, bsp_matrix_t* out) {
  if (!h || !out || n < 0 || bs < 1) return BSP_INVALID;
  *out = nullptr;
  BSP_CUDA_TRY(cudaSetDevice(h->device));
  std::vector<int> ptr(n + 1), col(n);
  for (int i = 0; i < n; ++i) {
    ptr[i + 1] = i + 1;
    col[i] = i;
  }
  bsp_matrix_t C = nullptr;
  BSP_TRY(make_matrix(h, n, n, bs, ptr, col, &C));
  if (n > 0)
    bsp::count_launch(), k_identity_blocks<<<grid_for(h, (int64_t)n * bs * bs, 256), 256, 0, h->stream>>>(
        n, bs, C->vals.get());
  BSP_CUDA_TRY(cudaPeekAtLastError());
  BSP_CUDA_TRY(cudaStreamSynchronize(h->stream));
  *out = C;
  return BSP_OK;
}

int bsp_bs_tr(bsp_handle_t h, bsp_matrix_t A, bsp_matrix_t* out) {
  if (!h || !A || !out) return BSP_INVALID;
  *out = nullptr;
  BSP_CUDA_TRY(cudaSetDevice(h->device));
  std::vector<int> ptr, col;
  std::vector<int64_t> src;
  transpose_struct(A, ptr, col, src);
  bsp_matrix_t C = nullptr;
  BSP_TRY(make_matrix(h, A->n_cols, A->n_rows, A->bs, ptr, col, &C));
  std::unique_ptr<bsp_matrix_s> guard(C);
  if (A->nnzb > 0) {
    DevBuf<int64_t> ds;
    BSP_TRY(upload_tmp(ds, src));
    bsp::count_launch(), k_block_combine<<<grid_for(h, A->nnzb * A->bs * A->bs, 256), 256, 0, h->stream>>>(
        A->nnzb, A->bs, ds.get(), nullptr, A->vals.get(), nullptr, 1.0, 0.0, 1, C->vals.get());
    BSP_CUDA_TRY(cudaPeekAtLastError());
    BSP_CUDA_TRY(cudaStreamSynchronize(h->stream));
  }
  *out = guard.release();
  return BSP_OK;
}

int bsp_matrix_add(bsp_handle_t h, double alpha, bsp_matrix_t A, double beta, bsp_matrix_t B, bsp_matrix_t* out) {
  if (!h || !A || !B || !out) return BSP_INVALID;
  *out = nullptr;
  if (A->n_rows != B->n_rows || A->n_cols != B->n_cols || A->bs != B->bs) {
    record_error("bsp_matrix_add: matrices of different shape or block size");
    return BSP_INVALID;
  }
  BSP_CUDA_TRY(cudaSetDevice(h->device));
  // A's blocks in order, then B's blocks missing from A appended per row
  // (CSR::operator+=, blocksp_containers.hpp:302-309)
  const int m = A->n_rows;
  std::vector<int> ptr(m + 1, 0), col;
  std::vector<int64_t> ia, ib;
  std::vector<int> pos(A->n_cols, -1);
  for (int i = 0; i < m; ++i) {
    const int base = (int)col.size();
    for (int t = A->h_row_ptr[i]; t < A->h_row_ptr[i + 1]; ++t) {
      pos[A->h_col_idx[t]] = (int)col.size();
      col.push_back(A->h_col_idx[t]);
      ia.push_back(t);
      ib.push_back(-1);
    }
    for (int t = B->h_row_ptr[i]; t < B->h_row_ptr[i + 1]; ++t) {
      const int j = B->h_col_idx[t];
      if (pos[j] >= base) {
        ib[pos[j]] = t;
      } else {
        pos[j] = (int)col.size();
        col.push_back(j);
        ia.push_back(-1);
        ib.push_back(t);
      }
    }
    for (int e = base; e < (int)col.size(); ++e) pos[col[e]] = -1;
    ptr[i + 1] = (int)col.size();
  }
  bsp_matrix_t C = nullptr;
  BSP_TRY(make_matrix(h, m, A->n_cols, A->bs, ptr, col, &C));
  std::unique_ptr<bsp_matrix_s> guard(C);
  if (!col.empty()) {
    DevBuf<int64_t> da, db;
    BSP_TRY(upload_tmp(da, ia));
    BSP_TRY(upload_tmp(db, ib));
    bsp::count_launch(), k_block_combine<<<grid_for(h, (int64_t)col.size() * A->bs * A->bs, 256), 256, 0,
                                           h->stream>>>((int64_t)col.size(), A->bs, da.get(), db.get(),
                                                        A->vals.get(), B->vals.get(), alpha, beta, 0,
                                                        C->vals.get());
    BSP_CUDA_TRY(cudaPeekAtLastError());
    BSP_CUDA_TRY(cudaStreamSynchronize(h->stream));
  }
  *out = guard.release();
  return BSP_OK;
}

int bsp_bsmm(bsp_handle_t h, bsp_matrix_t A, bsp_matrix_t B, int a_transpose, bsp_matrix_t* out) {
  if (!h || !A || !B || !out) return BSP_INVALID;
  *out = nullptr;
  if (A->bs != B->bs || A->bs > 32) {
    record_error("bsp_bsmm: block sizes differ or exceed 32");
    return BSP_INVALID;
  }
  if ((a_transpose ? A->n_rows : A->n_cols) != B->n_rows) {
    record_error("bsp_bsmm: inner dimensions differ");
    return BSP_INVALID;
  }
  BSP_CUDA_TRY(cudaSetDevice(h->device));
  // op(A) as a matrix of its own when transposed
  bsp_matrix_t At = nullptr;
  if (a_transpose) BSP_TRY(bsp_bs_tr(h, A, &At));
  std::unique_ptr<bsp_matrix_s> at_guard(At);
  const bsp_matrix_s* L = a_transpose ? At : A;
  const int m = L->n_rows, nc = B->n_cols, bs = A->bs;
  // structure: blocks of row i in order of first creation; pairs per block
  std::vector<int> ptr(m + 1, 0), col, mark(nc, -1), slot(nc, 0);
  std::vector<int64_t> pair_cnt;
  std::vector<std::pair<int64_t, std::pair<int, int>>> pairs;  // (C block, (a, b)) in order of addition
  for (int i = 0; i < m; ++i) {
    for (int a = L->h_row_ptr[i]; a < L->h_row_ptr[i + 1]; ++a) {
      const int k = L->h_col_idx[a];
      for (int b = B->h_row_ptr[k]; b < B->h_row_ptr[k + 1]; ++b) {
        const int j = B->h_col_idx[b];
        if (mark[j] != i) {
          mark[j] = i;
          slot[j] = (int)col.size();
          col.push_back(j);
          pair_cnt.push_back(0);
        }
        pair_cnt[slot[j]]++;
        pairs.push_back({slot[j], {a, b}});
      }
    }
    ptr[i + 1] = (int)col.size();
  }
  const int64_t ncb = (int64_t)col.size();
  std::vector<int64_t> pair_ptr(ncb + 1, 0);
  for (int64_t c = 0; c < ncb; ++c) pair_ptr[c + 1] = pair_ptr[c] + pair_cnt[c];
  std::vector<int> pa(pairs.size()), pb(pairs.size());
  {
    std::vector<int64_t> fill(pair_ptr.begin(), pair_ptr.end() - 1);
    for (auto& p : pairs) {  // stable: pairs of one C block keep their order of addition
      const int64_t at = fill[p.first]++;
      pa[at] = p.second.first;
      pb[at] = p.second.second;
    }
  }
  bsp_matrix_t C = nullptr;
  BSP_TRY(make_matrix(h, m, nc, bs, ptr, col, &C));
  std::unique_ptr<bsp_matrix_s> guard(C);
  if (ncb > 0) {
    DevBuf<int64_t> dptr;
    DevBuf<int> dpa, dpb;
    BSP_TRY(upload_tmp(dptr, pair_ptr));
    BSP_TRY(upload_tmp(dpa, pa));
    BSP_TRY(upload_tmp(dpb, pb));
    const size_t smem = (size_t)kMMWarps * 2 * bs * bs * sizeof(double);
    BSP_CUDA_TRY(cudaFuncSetAttribute(k_bsmm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int grid = (int)std::min<int64_t>((ncb + kMMWarps - 1) / kMMWarps, (int64_t)h->num_sms * 16);
    bsp::count_launch(), k_bsmm<<<grid, kMMWarps * 32, smem, h->stream>>>(ncb, bs, dptr.get(), dpa.get(), dpb.get(),
                                                                           L->vals.get(), B->vals.get(),
                                                                           C->vals.get());
    BSP_CUDA_TRY(cudaPeekAtLastError());
    BSP_CUDA_TRY(cudaStreamSynchronize(h->stream));
  }
  *out = guard.release();
  return BSP_OK;
}

int bsp_matrix_export(bsp_matrix_t A, int* row_ptr, int* col_idx, double* vals) {
  if (!A || !row_ptr || !col_idx || !vals) return BSP_INVALID;
  BSP_CUDA_TRY(cudaSetDevice(A->device));
  std::copy(A->h_row_ptr.begin(), A->h_row_ptr.end(), row_ptr);
  std::copy(A->h_col_idx.begin(), A->h_col_idx.end(), col_idx);
  if (A->nnzb > 0)
    BSP_CUDA_TRY(cudaMemcpy(vals, A->vals.get(), (size_t)A->nnzb * A->bs * A->bs * sizeof(double),
                            cudaMemcpyDeviceToHost));
  return BSP_OK;
}

}  // extern "C"
