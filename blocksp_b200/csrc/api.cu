// api.cu — C ABI glue: handles, matrices, bsmv and vector reductions.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <map>
#include <mutex>
#include "reduce.cuh"

namespace bsp {

static thread_local std::string g_last_error;
void record_error(const std::string& msg) { g_last_error = msg; }

// ---- device memory cache (see pool_alloc in internal.hpp) ----
namespace {
struct Pool {
  std::mutex mu;
  std::map<int, std::multimap<size_t, void*>> free_blocks;  // device -> (capacity, block)
  std::map<int, size_t> cached;                             // device -> bytes held
};
// Never destroyed: buffers released during static destruction still find it.
Pool& pool() {
  static Pool* p = new Pool;
  return *p;
}
void pool_trim_locked(Pool& P, int device) {
  for (auto& kv : P.free_blocks) {
    if (device >= 0 && kv.first != device) continue;
    int cur = -1;
    cudaGetDevice(&cur);
    if (cur != kv.first) cudaSetDevice(kv.first);
    for (auto& b : kv.second) cudaFree(b.second);
    kv.second.clear();
    P.cached[kv.first] = 0;
    if (cur >= 0 && cur != kv.first) cudaSetDevice(cur);
  }
}
}  // namespace

cudaError_t pool_alloc(void** p, size_t bytes, size_t* cap, int* device) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  *device = dev;
  Pool& P = pool();
  {
    std::lock_guard<std::mutex> lk(P.mu);
    auto& fl = P.free_blocks[dev];
    auto it = fl.lower_bound(bytes);
    // a cached block at most 1/8 (plus 1 MiB) larger than the request
    if (it != fl.end() && it->first <= bytes + bytes / 8 + (size_t(1) << 20)) {
      *p = it->second;
      *cap = it->first;
      P.cached[dev] -= it->first;
      fl.erase(it);
      return cudaSuccess;
    }
  }
  e = cudaMalloc(p, bytes);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    {
      std::lock_guard<std::mutex> lk(P.mu);
      pool_trim_locked(P, dev);
    }
    e = cudaMalloc(p, bytes);
  }
  *cap = bytes;
  return e;
}

void pool_free(void* p, size_t cap, int device) {
  int cur = -1;
  cudaGetDevice(&cur);
  if (device >= 0 && cur != device) cudaSetDevice(device);
  // queued work may still use the block: wait as cudaFree does
  const bool idle = cudaDeviceSynchronize() == cudaSuccess;
  Pool& P = pool();
  {
    std::lock_guard<std::mutex> lk(P.mu);
    if (idle && P.cached[device] + cap <= kPoolMaxBytes) {
      P.free_blocks[device].emplace(cap, p);
      P.cached[device] += cap;
      p = nullptr;
    }
  }
  if (p) cudaFree(p);
  if (cur >= 0 && device >= 0 && cur != device) cudaSetDevice(cur);
}

// ---- pattern registry (see SymbolicSet in internal.hpp) ----
namespace {
struct PatternEntry {
  int device = 0, n_rows = 0, n_cols = 0, bs = 0;
  int64_t nnzb = 0;
  uint64_t hash = 0;
  std::vector<int> row_ptr, col_idx;
  std::shared_ptr<SymbolicSet> set;
};
constexpr size_t kPatternsKept = 4;
std::mutex g_pat_mu;
std::vector<PatternEntry>* g_patterns = new std::vector<PatternEntry>;  // most recent last; never destroyed

uint64_t pattern_hash(int n_rows, int64_t nnzb, const int* rp, const int* ci) {
  uint64_t h = 0x9E3779B97F4A7C15ull ^ ((uint64_t)n_rows << 32) ^ (uint64_t)nnzb;
  auto mix = [&h](uint32_t v) {
    h ^= v;
    h *= 0xBF58476D1CE4E5B9ull;
    h ^= h >> 29;
  };
  for (int i = 0; i <= n_rows; ++i) mix((uint32_t)rp[i]);
  for (int64_t t = 0; t < nnzb; ++t) mix((uint32_t)ci[t]);
  return h;
}
}  // namespace

std::shared_ptr<SymbolicSet> symbolic_for_pattern(int device, int n_rows, int n_cols, int bs, int64_t nnzb,
                                                  const int* row_ptr, const int* col_idx) {
  const uint64_t h = pattern_hash(n_rows, nnzb, row_ptr, col_idx);
  std::lock_guard<std::mutex> lk(g_pat_mu);
  auto& P = *g_patterns;
  for (size_t k = 0; k < P.size(); ++k) {
    PatternEntry& e = P[k];
    if (e.device == device && e.n_rows == n_rows && e.n_cols == n_cols && e.bs == bs && e.nnzb == nnzb &&
        e.hash == h && std::equal(row_ptr, row_ptr + n_rows + 1, e.row_ptr.begin()) &&
        std::equal(col_idx, col_idx + nnzb, e.col_idx.begin())) {
      PatternEntry hit = std::move(e);
      P.erase(P.begin() + k);
      std::shared_ptr<SymbolicSet> set = hit.set;
      P.push_back(std::move(hit));
      return set;
    }
  }
  PatternEntry e;
  e.device = device;
  e.n_rows = n_rows;
  e.n_cols = n_cols;
  e.bs = bs;
  e.nnzb = nnzb;
  e.hash = h;
  e.row_ptr.assign(row_ptr, row_ptr + n_rows + 1);
  e.col_idx.assign(col_idx, col_idx + nnzb);
  e.set = std::make_shared<SymbolicSet>();
  std::shared_ptr<SymbolicSet> set = e.set;
  P.push_back(std::move(e));
  if (P.size() > kPatternsKept) P.erase(P.begin());
  return set;
}

void symbolic_registry_clear() {
  std::lock_guard<std::mutex> lk(g_pat_mu);
  g_patterns->clear();
}

static std::atomic<uint64_t> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void count_launch_add(int64_t n) { g_launches.fetch_add((uint64_t)n, std::memory_order_relaxed); }

int bsmv_launch(bsp_matrix_s* A, int nrhs, int transpose, int dtype, double alpha,
                const void* x, double beta, const void* z, void* y, cudaStream_t s);

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

static int check_device_present() {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    cudaGetLastError();
    record_error("no CUDA device visible: the BlockSp B200 path has no CPU fallback");
    return BSP_NO_DEVICE;
  }
  return BSP_OK;
}

static int validate_structure(int n_rows, int n_cols, int bs, int64_t nnzb, const int* row_ptr,
                              const int* col_idx) {
  if (n_rows < 0 || n_cols < 0 || bs < 1 || bs > 64 || nnzb < 0) {
    record_error("matrix: bad sizes");
    return BSP_INVALID;
  }
  if (!row_ptr || (nnzb > 0 && !col_idx)) {
    record_error("matrix: null structure pointer");
    return BSP_INVALID;
  }
  if (row_ptr[0] != 0 || row_ptr[n_rows] != nnzb) {
    record_error("matrix: row_ptr must start at 0 and end at nnzb");
    return BSP_INVALID;
  }
  if (nnzb > INT32_MAX) {
    record_error("matrix: more than 2^31-1 blocks");
    return BSP_INVALID;
  }
  // One O(nnzb) pass: range checks, and duplicate columns within a row (not
  // representable in the reference container: operator() finds the existing
  // entry, containers.hpp:156-157) found with a per-column stamp of the last
  // row that used it, so no row is copied or sorted.
  std::vector<int> stamp(n_cols, -1);
  for (int i = 0; i < n_rows; ++i) {
    if (row_ptr[i + 1] < row_ptr[i]) {
      record_error("matrix: row_ptr not monotone");
      return BSP_INVALID;
    }
    for (int t = row_ptr[i]; t < row_ptr[i + 1]; ++t) {
      const int c = col_idx[t];
      if (c < 0 || c >= n_cols) {
        record_error("matrix: column index out of range in row " + std::to_string(i));
        return BSP_INVALID;
      }
      if (stamp[c] == i) {
        record_error("matrix: duplicate column in row " + std::to_string(i));
        return BSP_INVALID;
      }
      stamp[c] = i;
    }
  }
  return BSP_OK;
}

}  // namespace bsp

using namespace bsp;

extern "C" {

int bsp_abi_version(void) { return BSP_ABI_VERSION; }

uint64_t bsp_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

const char* bsp_status_string(int s) {
  switch (s) {
    case BSP_OK: return "ok";
    case BSP_ZERO_PIVOT: return "zero pivot in a diagonal block";
    case BSP_NOT_SPD: return "block Cholesky met a non-positive pivot";
    case BSP_BREAKDOWN: return "Krylov breakdown";
    case BSP_MAXIT: return "maximum iterations reached";
    case BSP_NAN: return "NaN or Inf in residual";
    case BSP_TIMEOUT: return "bounded device wait timed out";
    case BSP_CUDA_ERROR: return "CUDA error";
    case BSP_INVALID: return "invalid argument";
    case BSP_NO_DEVICE: return "no CUDA device";
    case BSP_OUT_OF_MEMORY: return "out of device memory";
    default: return "unknown status";
  }
}

const char* bsp_last_error(bsp_handle_t h) {
  if (h) {
    h->last_error = g_last_error;
    return h->last_error.c_str();
  }
  return g_last_error.c_str();
}

int bsp_device_count(int* count) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess) {
    cudaGetLastError();
    n = 0;
  }
  if (count) *count = n;
  return n > 0 ? BSP_OK : BSP_NO_DEVICE;
}

int bsp_handle_create(int device, void* stream, bsp_handle_t* out) {
  if (!out) return BSP_INVALID;
  *out = nullptr;
  BSP_TRY(check_device_present());
  BSP_CUDA_TRY(cudaSetDevice(device));
  auto h = std::make_unique<bsp_handle_s>();
  h->device = device;
  cudaDeviceProp prop;
  BSP_CUDA_TRY(cudaGetDeviceProperties(&prop, device));
  h->num_sms = prop.multiProcessorCount;
  if (stream) {
    h->stream = (cudaStream_t)stream;
  } else {
    BSP_CUDA_TRY(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    h->own_stream = true;
  }
  BSP_TRY(h->ws.partials.alloc((size_t)kRedSlots * kRedBlocks * 4));
  BSP_TRY(h->ws.tickets.alloc(kRedSlots));
  BSP_TRY(h->ws.scalars.alloc(256));
  BSP_TRY(h->ws.status.alloc(1));
  BSP_CUDA_TRY(cudaMemset(h->ws.tickets.get(), 0, kRedSlots * sizeof(unsigned)));
  BSP_CUDA_TRY(cudaMemset(h->ws.scalars.get(), 0, 256 * sizeof(double)));
  BSP_CUDA_TRY(cudaMemset(h->ws.status.get(), 0, sizeof(DevStatus)));
  *out = h.release();
  return BSP_OK;
}

int bsp_release_cached_memory(int device) {
  symbolic_registry_clear();  // its analyses hold device buffers too
  Pool& P = pool();
  std::lock_guard<std::mutex> lk(P.mu);
  pool_trim_locked(P, device);
  return BSP_OK;
}

int bsp_cached_memory(int device, int64_t* bytes) {
  if (!bytes) return BSP_INVALID;
  Pool& P = pool();
  std::lock_guard<std::mutex> lk(P.mu);
  *bytes = (int64_t)P.cached[device];
  return BSP_OK;
}

int bsp_handle_set_spin_limit(bsp_handle_t h, unsigned polls) {
  if (!h || polls < 1) return BSP_INVALID;
  h->spin_limit = polls;
  return BSP_OK;
}

int bsp_handle_destroy(bsp_handle_t h) {
  if (!h) return BSP_OK;
  {
    DeviceGuard g(h->device);
    cudaStreamSynchronize(h->stream);
    h->ws = Workspace{};
    if (h->own_stream) cudaStreamDestroy(h->stream);
  }
  delete h;
  return BSP_OK;
}

int bsp_handle_sync(bsp_handle_t h) {
  if (!h) return BSP_INVALID;
  DeviceGuard g(h->device);
  BSP_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return BSP_OK;
}

void* bsp_handle_stream(bsp_handle_t h) { return h ? (void*)h->stream : nullptr; }

// pre_vals: the value buffer, already allocated (and being filled) by the
// caller; null: allocate it here.
static int matrix_create_common(bsp_handle_t h, int n_rows, int n_cols, int bs, int64_t nnzb,
                                const int* row_ptr, const int* col_idx, bsp_matrix_t* out,
                                std::unique_ptr<bsp_matrix_s>& A, DevBuf<double>* pre_vals = nullptr) {
  BSP_TRY(validate_structure(n_rows, n_cols, bs, nnzb, row_ptr, col_idx));
  A = std::make_unique<bsp_matrix_s>();
  A->h = h;
  A->device = h->device;
  A->n_rows = n_rows;
  A->n_cols = n_cols;
  A->bs = bs;
  A->nnzb = nnzb;
  A->h_row_ptr.assign(row_ptr, row_ptr + n_rows + 1);
  A->h_col_idx.assign(col_idx, col_idx + nnzb);
  A->sym = symbolic_for_pattern(h->device, n_rows, n_cols, bs, nnzb, row_ptr, col_idx);
  BSP_TRY(A->row_ptr.alloc(n_rows + 1));
  BSP_TRY(A->col_idx.alloc(nnzb > 0 ? nnzb : 1));
  if (pre_vals) A->vals = std::move(*pre_vals);
  else BSP_TRY(A->vals.alloc(nnzb > 0 ? (size_t)nnzb * bs * bs : 1));
  BSP_CUDA_TRY(cudaMemcpy(A->row_ptr.get(), row_ptr, (n_rows + 1) * sizeof(int), cudaMemcpyHostToDevice));
  if (nnzb > 0)
    BSP_CUDA_TRY(cudaMemcpy(A->col_idx.get(), col_idx, nnzb * sizeof(int), cudaMemcpyHostToDevice));
  (void)out;
  return BSP_OK;
}

int bsp_matrix_create(bsp_handle_t h, int n_rows, int n_cols, int bs, int64_t nnzb,
                      const int* row_ptr, const int* col_idx, const double* vals,
                      bsp_matrix_t* out) {
  if (!h || !out) return BSP_INVALID;
  *out = nullptr;
  DeviceGuard g(h->device);
  if (n_rows < 0 || bs < 1 || bs > 64 || nnzb < 0 || nnzb > INT32_MAX || (nnzb > 0 && !vals)) {
    record_error("matrix: bad sizes or null values");
    return BSP_INVALID;
  }
  // The values travel (asynchronously from pinned memory) while the host
  // validates and registers the structure.
  DevBuf<double> dv;
  BSP_TRY(dv.alloc(nnzb > 0 ? (size_t)nnzb * bs * bs : 1));
  if (nnzb > 0)
    BSP_CUDA_TRY(cudaMemcpyAsync(dv.get(), vals, (size_t)nnzb * bs * bs * sizeof(double), cudaMemcpyHostToDevice,
                                 h->stream));
  std::unique_ptr<bsp_matrix_s> A;
  const int st = matrix_create_common(h, n_rows, n_cols, bs, nnzb, row_ptr, col_idx, out, A, &dv);
  // the copy ends before any buffer is released or handed out
  const cudaError_t se = cudaStreamSynchronize(h->stream);
  if (st != BSP_OK) return st;
  if (se != cudaSuccess) {
    record_error(std::string("matrix upload: ") + cudaGetErrorString(se));
    return BSP_CUDA_ERROR;
  }
  *out = A.release();
  return BSP_OK;
}

int bsp_matrix_create_dev(bsp_handle_t h, int n_rows, int n_cols, int bs, int64_t nnzb,
                          const int* d_row_ptr, const int* d_col_idx, const double* d_vals,
                          bsp_matrix_t* out) {
  if (!h || !out) return BSP_INVALID;
  *out = nullptr;
  DeviceGuard g(h->device);
  if (n_rows < 0 || nnzb < 0) return BSP_INVALID;
  std::vector<int> rp(n_rows + 1), ci(nnzb);
  BSP_CUDA_TRY(cudaMemcpy(rp.data(), d_row_ptr, (n_rows + 1) * sizeof(int), cudaMemcpyDeviceToHost));
  if (nnzb > 0)
    BSP_CUDA_TRY(cudaMemcpy(ci.data(), d_col_idx, nnzb * sizeof(int), cudaMemcpyDeviceToHost));
  std::unique_ptr<bsp_matrix_s> A;
  BSP_TRY(matrix_create_common(h, n_rows, n_cols, bs, nnzb, rp.data(), ci.data(), out, A));
  if (nnzb > 0)
    BSP_CUDA_TRY(cudaMemcpy(A->vals.get(), d_vals, (size_t)nnzb * bs * bs * sizeof(double),
                            cudaMemcpyDeviceToDevice));
  *out = A.release();
  return BSP_OK;
}

int bsp_matrix_destroy(bsp_matrix_t A) {
  // Does not touch A->h: the handle may already be gone.  cudaFree in the
  // buffer destructors synchronises the device before releasing memory.
  if (!A) return BSP_OK;
  DeviceGuard g(A->device);
  delete A;
  return BSP_OK;
}

int bsp_matrix_info(bsp_matrix_t A, int* n_rows, int* n_cols, int* bs, int64_t* nnzb) {
  if (!A) return BSP_INVALID;
  if (n_rows) *n_rows = A->n_rows;
  if (n_cols) *n_cols = A->n_cols;
  if (bs) *bs = A->bs;
  if (nnzb) *nnzb = A->nnzb;
  return BSP_OK;
}

int bsp_matrix_device_ptrs(bsp_matrix_t A, const int** row_ptr, const int** col_idx,
                           const double** vals) {
  if (!A) return BSP_INVALID;
  if (row_ptr) *row_ptr = A->row_ptr.get();
  if (col_idx) *col_idx = A->col_idx.get();
  if (vals) *vals = A->vals.get();
  return BSP_OK;
}

}  // extern "C"

int matrix_create_struct(bsp_handle_t h, int n_rows, int n_cols, int bs, int64_t nnzb, const int* row_ptr,
                         const int* col_idx, bsp_matrix_t* out) {
  std::unique_ptr<bsp_matrix_s> A;
  BSP_TRY(matrix_create_common(h, n_rows, n_cols, bs, nnzb, row_ptr, col_idx, out, A));
  *out = A.release();
  return BSP_OK;
}

namespace bsp {
__global__ void k_to_f32(int64_t n, const double* __restrict__ a, float* __restrict__ b) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}
__global__ void k_to_bf16(int64_t n, const double* __restrict__ a, __nv_bfloat16* __restrict__ b) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    b[i] = __float2bfloat16_rn((float)a[i]);  // double -> float -> bf16, both round-to-nearest-even
}
__global__ void k_axpy(int64_t n, double a, const double* __restrict__ x, double* __restrict__ y) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    y[i] = fma(a, x[i], y[i]);
}
int grid_for(const bsp_handle_s* h, int64_t n, int threads) {
  int64_t g = ceil_div(n, threads);
  int64_t cap = (int64_t)h->num_sms * 8;
  return (int)std::max<int64_t>(1, std::min(g, cap));
}
}  // namespace bsp

extern "C" {

int bsp_matrix_make_lowp(bsp_matrix_t A, int dtype) {
  if (!A) return BSP_INVALID;
  DeviceGuard g(A->h->device);
  const int64_t n = A->nnzb * A->bs * A->bs;
  if (dtype == BSP_F32) {
    if (A->vals32.get()) return BSP_OK;
    BSP_TRY(A->vals32.alloc(n > 0 ? n : 1));
    if (n > 0) bsp::count_launch(), k_to_f32<<<grid_for(A->h, n, 256), 256, 0, A->h->stream>>>(n, A->vals.get(), A->vals32.get());
  } else if (dtype == BSP_BF16) {
    if (A->vals16.get()) return BSP_OK;
    BSP_TRY(A->vals16.alloc(n > 0 ? n : 1));
    if (n > 0) bsp::count_launch(), k_to_bf16<<<grid_for(A->h, n, 256), 256, 0, A->h->stream>>>(n, A->vals.get(), A->vals16.get());
  } else if (dtype != BSP_F64) {
    return BSP_INVALID;
  }
  BSP_CUDA_TRY(cudaPeekAtLastError());
  return BSP_OK;
}

int bsp_bsmv_dev(bsp_handle_t h, bsp_matrix_t A, int nrhs, int transpose, int dtype,
                 double alpha, const void* x, double beta, const void* z, void* y) {
  if (!h || !A || !x || !y) return BSP_INVALID;
  if (beta != 0.0 && !z) return BSP_INVALID;
  DeviceGuard g(h->device);
  return bsmv_launch(A, nrhs, transpose, dtype, alpha, x, beta, z, y, h->stream);
}

int bsp_bsmv(bsp_handle_t h, bsp_matrix_t A, int nrhs, int transpose, double alpha,
             const double* x, double beta, double* y) {
  if (!h || !A || !x || !y) return BSP_INVALID;
  DeviceGuard g(h->device);
  const int64_t nx = (int64_t)(transpose ? A->n_rows : A->n_cols) * A->bs * nrhs;
  const int64_t ny = (int64_t)(transpose ? A->n_cols : A->n_rows) * A->bs * nrhs;
  BSP_TRY(h->stage(nx > 0 ? nx : 1, ny > 0 ? ny : 1));
  double* dx = h->stage_in.get();
  double* dy = h->stage_out.get();
  BSP_CUDA_TRY(cudaMemcpyAsync(dx, x, nx * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  if (beta != 0.0)
    BSP_CUDA_TRY(cudaMemcpyAsync(dy, y, ny * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  BSP_TRY(bsmv_launch(A, nrhs, transpose, BSP_F64, alpha, dx, beta, dy, dy, h->stream));
  BSP_CUDA_TRY(cudaMemcpyAsync(y, dy, ny * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  BSP_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return BSP_OK;
}

int bsp_dot_dev(bsp_handle_t h, int64_t n, const double* x, const double* y, double* out_dev) {
  if (!h || n < 0 || !out_dev) return BSP_INVALID;
  DeviceGuard g(h->device);
  return launch_reduce<1>(h, 0, n, DotBody{x, y}, StoreFin{out_dev});
}

int bsp_dot(bsp_handle_t h, int64_t n, const double* x_dev, const double* y_dev, double* out_host) {
  if (!out_host) return BSP_INVALID;
  BSP_TRY(bsp_dot_dev(h, n, x_dev, y_dev, h->ws.scalars.get()));
  BSP_CUDA_TRY(cudaMemcpyAsync(out_host, h->ws.scalars.get(), sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  BSP_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return BSP_OK;
}

int bsp_axpy_dev(bsp_handle_t h, int64_t n, double a, const double* x, double* y) {
  if (!h || n < 0) return BSP_INVALID;
  DeviceGuard g(h->device);
  if (n == 0) return BSP_OK;
  bsp::count_launch(), k_axpy<<<grid_for(h, n, 256), 256, 0, h->stream>>>(n, a, x, y);
  BSP_CUDA_TRY(cudaPeekAtLastError());
  return BSP_OK;
}

}  // extern "C"
