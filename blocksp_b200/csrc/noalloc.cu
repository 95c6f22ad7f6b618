// noalloc.cu — FP64 dot product for callers that cannot allocate device memory.
//
// bsp_dot_dev needs a handle, and creating a handle allocates its reduction
// workspace with cudaMalloc.  Some callers cannot do that at the point where
// they need a dot product: code running while another framework owns the
// device allocator (plugins and callbacks that are handed a stream and device
// pointers but may not allocate), or code on a path where an allocation
// would synchronise the device or fail under a memory cap.  bsp_dot_noalloc
// serves them: it takes a stream and device pointers and allocates nothing.
//
// Its scratch (one partial sum per CTA plus the last-CTA ticket) lives in a
// file-scope __device__ array of fixed size.  Every GPU that loads this
// library holds that array (about 32 KiB) until the process exits.  The
// kernel is the same deterministic reduction as bsp_dot_dev (k_reduce with a
// dot body); here the grid is one CTA per kNoAllocChunk elements, so the
// largest n is kNoAllocMaxN = 33,554,432 elements.
#include <mutex>
#include "reduce.cuh"

namespace bsp {

constexpr int kNoAllocChunk = kRedThreads * 16;           // 8,192 elements per CTA
constexpr int kNoAllocMaxBlocks = 4096;                   // partial sums held in scratch
constexpr int64_t kNoAllocMaxN = (int64_t)kNoAllocChunk * kNoAllocMaxBlocks;
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_partials[kNoAllocMaxBlocks];
static __device__ __align__(256) unsigned g_noalloc_ticket[64];  // [0] is the ticket

namespace {
struct ScratchAddr {
  double* partials = nullptr;
  unsigned* ticket = nullptr;
  bool ready = false;
};
ScratchAddr g_addr[kNoAllocMaxDevices];
std::mutex g_addr_mu;

// The names above are host-side stand-ins; the kernel needs the device
// addresses, resolved once per device with that device current.  They stay
// cached until exit, so they are stale after a cudaDeviceReset of that device
// (the header says so: no calls on a device after resetting it).
int scratch_for_current_device(ScratchAddr* out) {
  int dev = 0;
  BSP_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocMaxDevices) {
    record_error("bsp_dot_noalloc: device index beyond the supported range");
    return BSP_INVALID;
  }
  std::lock_guard<std::mutex> lk(g_addr_mu);
  ScratchAddr& a = g_addr[dev];
  if (!a.ready) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
    if (e != cudaSuccess) {
      record_error(std::string("bsp_dot_noalloc: cudaGetSymbolAddress(partials): ") + cudaGetErrorString(e));
      return BSP_CUDA_ERROR;
    }
    a.partials = static_cast<double*>(p);
    e = cudaGetSymbolAddress(&p, g_noalloc_ticket);
    if (e != cudaSuccess) {
      record_error(std::string("bsp_dot_noalloc: cudaGetSymbolAddress(ticket): ") + cudaGetErrorString(e));
      return BSP_CUDA_ERROR;
    }
    a.ticket = static_cast<unsigned*>(p);
    a.ready = true;
  }
  *out = a;
  return BSP_OK;
}
}  // namespace

}  // namespace bsp

using namespace bsp;

extern "C" int bsp_dot_noalloc(void* stream, int64_t n, const double* x, const double* y,
                               double* out_dev) {
  if (n < 0 || !out_dev || (n > 0 && (!x || !y))) {
    record_error("bsp_dot_noalloc: bad argument");
    return BSP_INVALID;
  }
  if (n > kNoAllocMaxN) {
    record_error("bsp_dot_noalloc: n = " + std::to_string(n) + " exceeds the maximum of " +
                 std::to_string(kNoAllocMaxN) + " elements that its fixed scratch supports");
    return BSP_INVALID;
  }
  ScratchAddr a;
  BSP_TRY(scratch_for_current_device(&a));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // the ticket must start at zero; the partials are written before being read
  BSP_CUDA_TRY(cudaMemsetAsync(a.ticket, 0, sizeof(unsigned), s));
  const int blocks = (int)std::max<int64_t>(1, ceil_div(n, kNoAllocChunk));
  bsp::count_launch(), k_reduce<1, DotBody, StoreFin><<<blocks, kRedThreads, 0, s>>>(n, DotBody{x, y}, StoreFin{out_dev},
                                                                 a.partials, a.ticket);
  BSP_CUDA_TRY(cudaPeekAtLastError());
  return BSP_OK;
}
