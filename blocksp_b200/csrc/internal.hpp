// internal.hpp — host-side objects behind the C ABI handles.
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <vector>
#include "common.cuh"

namespace bsp {

// Process-wide cache of device allocations, per device.  A freed block is
// kept (after the device has finished all queued work, as cudaFree would
// wait) and handed to a later allocation of nearly the same size, so building
// matrices and preconditioners repeatedly does not pay cudaMalloc / cudaFree
// for gigabytes each time.  At most kPoolMaxBytes are kept per device; an
// allocation that fails frees the cache and retries; bsp_release_cached_memory
// returns it to the driver.
constexpr size_t kPoolMaxBytes = size_t(32) << 30;
cudaError_t pool_alloc(void** p, size_t bytes, size_t* cap, int* device);
void pool_free(void* p, size_t cap, int device);

// Owning device buffer: plain device memory (no stream-ordered allocator), so
// the pointers stay valid across streams and graph captures.  cap is the
// size of the underlying block in bytes (at least n * sizeof(T)).
template <typename T> struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  size_t cap = 0;
  int dev = -1;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n), cap(o.cap), dev(o.dev) { o.p = nullptr; o.n = o.cap = 0; }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      release();
      p = o.p; n = o.n; cap = o.cap; dev = o.dev;
      o.p = nullptr; o.n = o.cap = 0;
    }
    return *this;
  }
  ~DevBuf() { release(); }
  void release() {
    if (p) pool_free(p, cap, dev);
    p = nullptr;
    n = cap = 0;
  }
  int alloc(size_t count) {
    release();
    if (count == 0) return BSP_OK;
    void* q = nullptr;
    cudaError_t e = pool_alloc(&q, count * sizeof(T), &cap, &dev);
    if (e != cudaSuccess) {
      p = nullptr;
      cap = 0;
      record_error(std::string("cudaMalloc: ") + cudaGetErrorString(e));
      return e == cudaErrorMemoryAllocation ? BSP_OUT_OF_MEMORY : BSP_CUDA_ERROR;
    }
    p = static_cast<T*>(q);
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

struct StreamSym;
struct FactorPlan;

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
  // streamed layouts of the two sweeps (block sizes the streamed kernel takes)
  std::shared_ptr<StreamSym> ss_lo, ss_up;
  // elimination plan of the row-resident factorisation kernel
  std::shared_ptr<FactorPlan> plan;
};

// The analyses of one sparsity pattern.  Matrices created with the same
// pattern on the same device share one set (a process-wide registry keeps the
// sets of the last few patterns), so a new matrix with a known pattern —
// a new time step, a Newton update — skips the host analysis.
struct SymbolicSet {
  SymbolicCache ilu, ichol, sor;
};
std::shared_ptr<SymbolicSet> symbolic_for_pattern(int device, int n_rows, int n_cols, int bs, int64_t nnzb,
                                                  const int* row_ptr, const int* col_idx);
void symbolic_registry_clear();

// Non-owning view of a scratch buffer (handle scratch; see bsp_handle_s).
template <typename T> struct Span {
  T* p = nullptr;
  T* get() const { return p; }
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
  // polls a device wait makes before it gives up with BSP_TIMEOUT
  unsigned spin_limit = bsp::kSpinLimit;
  // staging buffers of the host-buffer entry points (grow-only, reused)
  bsp::DevBuf<double> stage_in, stage_out;
  // Grow-only device scratch of the solvers, by purpose.  Every call on a
  // handle is stream-ordered (and the solvers return after their work), so a
  // buffer is free again when the next call that uses it is enqueued; reuse
  // avoids cudaMalloc/cudaFree (a device-wide synchronisation) per solve.
  std::map<std::string, bsp::DevBuf<unsigned char>> scratch_bufs;
  template <typename T> int scratch(const std::string& tag, size_t count, T** out) {
    auto& b = scratch_bufs[tag];
    const size_t bytes = (count ? count : 1) * sizeof(T);
    if (b.n < bytes) {
      const int st = b.alloc(bytes);
      if (st) return st;
    }
    *out = reinterpret_cast<T*>(b.p);
    return 0;
  }
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
  // complex matrix held as its real embedding (bs = 2 cbs); 0 for a real one
  int cbs = 0;
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
  // symbolic analyses for ILU0 (full pattern), IChol0 (lower pattern), SOR/Diag,
  // shared with every matrix of the same pattern on this device
  std::shared_ptr<bsp::SymbolicSet> sym;
  // device memory of destroyed preconditioners of this matrix, handed to the
  // next one built on it (factor copies, inverted diagonals, scratch)
  std::vector<bsp::DevBuf<unsigned char>> bin;
};

namespace bsp {
constexpr size_t kBinMax = 64;
// d <- count elements, from A's bin when a buffer of fitting size is there.
template <typename T> int take(bsp_matrix_s* A, DevBuf<T>& d, size_t count) {
  count = count ? count : 1;
  const size_t bytes = count * sizeof(T);
  int best = -1;
  for (size_t i = 0; i < A->bin.size(); ++i)
    if (A->bin[i].n >= bytes && A->bin[i].n <= 2 * bytes + (1u << 20) &&
        (best < 0 || A->bin[i].n < A->bin[best].n))
      best = (int)i;
  if (best < 0) return d.alloc(count);
  d.release();
  d.p = reinterpret_cast<T*>(A->bin[best].p);
  d.n = count;
  d.cap = A->bin[best].cap;
  d.dev = A->bin[best].dev;
  A->bin[best].p = nullptr;
  A->bin[best].n = A->bin[best].cap = 0;
  A->bin.erase(A->bin.begin() + best);
  return BSP_OK;
}
// Hands d's memory to A's bin (the caller has made sure no work uses it).
template <typename T> void give(bsp_matrix_s* A, DevBuf<T>& d) {
  if (!d.p) return;
  DevBuf<unsigned char> r;
  r.p = reinterpret_cast<unsigned char*>(d.p);
  r.n = d.n * sizeof(T);
  r.cap = d.cap;
  r.dev = d.dev;
  d.p = nullptr;
  d.n = d.cap = 0;
  A->bin.push_back(std::move(r));
  if (A->bin.size() > kBinMax) A->bin.erase(A->bin.begin());
}
}  // namespace bsp

// Uploads a validated structure and allocates (uninitialised) FP64 values.
int matrix_create_struct(bsp_handle_t h, int n_rows, int n_cols, int bs, int64_t nnzb, const int* row_ptr,
                         const int* col_idx, bsp_matrix_t* out);
