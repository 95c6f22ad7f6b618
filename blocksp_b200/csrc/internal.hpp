// internal.hpp — host-side objects behind the C ABI handles.
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>
#include "common.cuh"

namespace bsp {

// Owning device buffer (cudaMallocAsync-free: plain cudaMalloc so that the
// pointers stay valid across streams and graph captures).
template <typename T> struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) { release(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
    return *this;
  }
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  int alloc(size_t count) {
    release();
    if (count == 0) return BSP_OK;
    cudaError_t e = cudaMalloc(&p, count * sizeof(T));
    if (e != cudaSuccess) {
      p = nullptr;
      record_error(std::string("cudaMalloc: ") + cudaGetErrorString(e));
      return e == cudaErrorMemoryAllocation ? BSP_OUT_OF_MEMORY : BSP_CUDA_ERROR;
    }
    n = count;
    return BSP_OK;
  }
  T* get() const { return p; }
};

// Workspace for deterministic reductions: per-CTA partials plus a ticket.
constexpr int kRedBlocks = 2 * kB200SMs;  // CTAs of a reduction launch
constexpr int kRedSlots = 16;             // independent reduction slots

struct Workspace {
  DevBuf<double> partials;   // kRedSlots * kRedBlocks * 4
  DevBuf<unsigned> tickets;  // kRedSlots
  DevBuf<double> scalars;    // small device scalars (dot results etc.)
  DevBuf<DevStatus> status;  // device error word
};

// Structure-only analysis behind a preconditioner (sorted factor pattern,
// permutation, dependency levels, chain tasks).  It depends on the matrix
// pattern alone, so it is computed once per matrix and kind and reused by
// every later preconditioner built on the same matrix.
struct SymbolicCache {
  bool valid = false;
  int64_t f_nnzb = 0;
  int n_lev_lo = 0, n_lev_up = 0, n_task_lo = 0, n_task_up = 0;
  std::vector<int64_t> h_perm;
  DevBuf<int> f_ptr, f_col, f_diag, order_lo, order_up, task_lo_row, task_lo_len, task_up_row,
      task_up_len, t_ptr, t_row, a_diag;
  DevBuf<int64_t> d_perm, t_blk;
};

// Device time between construction and stop_ms() on one stream.
struct EventTimer {
  cudaEvent_t a = nullptr, b = nullptr;
  cudaStream_t s;
  explicit EventTimer(cudaStream_t st) : s(st) {
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, s);
  }
  double stop_ms() {
    float ms = 0;
    cudaEventRecord(b, s);
    cudaEventSynchronize(b);
    cudaEventElapsedTime(&ms, a, b);
    return ms;
  }
  ~EventTimer() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
};

}  // namespace bsp

struct bsp_handle_s {
  int device = 0;
  int num_sms = bsp::kB200SMs;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  bsp::Workspace ws;
  std::string last_error;
  int epoch = 0;  // sync-free sweep epoch (flags hold the epoch of their last write)
  // staging buffers of the host-buffer entry points (grow-only, reused)
  bsp::DevBuf<double> stage_in, stage_out;
  int stage(size_t n_in, size_t n_out) {
    if (stage_in.n < n_in) { int s = stage_in.alloc(n_in); if (s) return s; }
    if (stage_out.n < n_out) { int s = stage_out.alloc(n_out); if (s) return s; }
    return 0;
  }
};

struct bsp_matrix_s {
  bsp_handle_t h = nullptr;  // creating handle; must outlive every compute call on A
  int device = 0;
  int n_rows = 0, n_cols = 0, bs = 0;
  int64_t nnzb = 0;
  bsp::DevBuf<int> row_ptr, col_idx;
  bsp::DevBuf<double> vals;
  bsp::DevBuf<float> vals32;
  bsp::DevBuf<__nv_bfloat16> vals16;
  // host copies of the structure (level scheduling, lowTri, transposes)
  std::vector<int> h_row_ptr, h_col_idx;
  // transposed structure for op(A) = A^T, built on first use:
  // for block column j, entries t in [tr_ptr[j], tr_ptr[j+1]) give the block
  // row tr_row[t] and the block index tr_blk[t] in vals.
  bsp::DevBuf<int> tr_ptr, tr_row;
  bsp::DevBuf<int64_t> tr_blk;
  bool has_transpose = false;
  // symbolic analyses for ILU0 (full pattern), IChol0 (lower pattern), SOR/Diag
  bsp::SymbolicCache sym_ilu, sym_ichol, sym_sor;
};

// Uploads a validated structure and allocates (uninitialised) FP64 values.
int matrix_create_struct(bsp_handle_t h, int n_rows, int n_cols, int bs, int64_t nnzb, const int* row_ptr,
                         const int* col_idx, bsp_matrix_t* out);
