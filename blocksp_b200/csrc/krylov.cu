// krylov.cu — pCG and pGMRES with deflated restart on sm_100a.
//
// Reference: blocksp_solvers.hpp:51-105 (pCG), :107-136 (one_arnoldi),
// :156-295 (pGMRES), blocksp_deflated_restart.hpp:38-269 (Morgan GMRES-DR).
//
// All vectors, scalars, the Hessenberg matrix and its least-squares state
// live on the GPU in FP64.  Per iteration the host enqueues kernels and reads
// back one small status word; no vector or Hessenberg data crosses PCIe.
//   * dots/norms are deterministic fused grid reductions (reduce.cuh),
//   * the Arnoldi step is modified Gram-Schmidt with each axpy fused into the
//     next dot (j+2 passes for column j),
//   * the least-squares problem is kept in Givens-QR form and updated by one
//     column per iteration (the reference re-solves it with gels each time;
//     both give the minimiser of the same problem),
//   * the deflated restart (harmonic Ritz values, Schur form, selection,
//     invariant subspace, P_{k+1}, c_r, H_new) runs on one GPU warp in
//     small_dense.h (working set in shared memory), and Qn <- Qn P_{k+1} is a tall-skinny in-place kernel.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <type_traits>
#include <vector>
#include "reduce.cuh"
#include "stage.cuh"
#include "sentinel.cuh"
#include "small_dense.h"

struct bsp_precond_s;

namespace bsp {

int bsmv_launch(bsp_matrix_s* A, int nrhs, int transpose, int dtype, double alpha,
                const void* x, double beta, const void* z, void* y, cudaStream_t s);
int precond_apply(bsp_precond_s* pc, int precision, const void* r, void* z);
int precond_check_status(bsp_precond_s* pc);
int grid_for(const bsp_handle_s* h, int64_t n, int threads);

constexpr double kEps = 2.220446049250313e-16;

enum { DONE_RUNNING = 0, DONE_CONVERGED = 1, DONE_MAXIT = 2, DONE_BREAKDOWN = 3, DONE_NAN = 4 };

// Status word read back by the host every iteration.
struct KHead {
  int done;
  int j;          // current Arnoldi column (pGMRES) / iteration count (pCG)
  int tot;        // pGMRES totIters
  int keff;       // columns kept by the last deflated restart
  int n_hist;
  int restarted;
  int breakdown;
  int pad;
  double res0, tolerance, res, zero_thresh;
  // pCG scalars
  double rz, pAp, alpha, beta;
};

// ------------------------------------------------------------------ kernels
__global__ void k_copy(int64_t n, const double* __restrict__ a, double* __restrict__ b) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = a[i];
}
// q = v / *h unless |*h| < zero_thresh (breakdown: the reference does not
// extend the basis, blocksp_solvers.hpp:133)
__global__ void k_div(int64_t n, const double* __restrict__ v, const double* __restrict__ h,
                      const KHead* __restrict__ head, double* __restrict__ q) {
  const double d = *h;
  if (fabs(d) < head->zero_thresh) return;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    q[i] = v[i] / d;
}
// p = z + beta p
__global__ void k_cg_p(int64_t n, const double* __restrict__ z, const KHead* __restrict__ head,
                       double* __restrict__ p) {
  const double beta = head->beta;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = z[i] + beta * p[i];
}

// ---- 4-element chunks: the reduction bodies below take a chunk index c and
// handle elements 4c .. 4c+3 (fewer at the tail), issuing every load of the
// chunk before the arithmetic so that a read-modify-write of one vector does
// not serialise the loads of the next elements behind it.
constexpr int kC = 4;
inline int64_t chunks_of(int64_t n) { return (n + kC - 1) / kC; }

struct V4 {
  double v[kC];
};
__device__ __forceinline__ V4 ld4(const double* p, int64_t e, int64_t n) {
  V4 r;
  if (e + kC <= n) {
    const double2 a = *reinterpret_cast<const double2*>(p + e);
    const double2 b = *reinterpret_cast<const double2*>(p + e + 2);
    r.v[0] = a.x; r.v[1] = a.y; r.v[2] = b.x; r.v[3] = b.y;
  } else {
#pragma unroll
    for (int k = 0; k < kC; ++k) r.v[k] = (e + k < n) ? p[e + k] : 0.0;
  }
  return r;
}
__device__ __forceinline__ void st4(double* p, int64_t e, int64_t n, const V4& r) {
  if (e + kC <= n) {
    *reinterpret_cast<double2*>(p + e) = make_double2(r.v[0], r.v[1]);
    *reinterpret_cast<double2*>(p + e + 2) = make_double2(r.v[2], r.v[3]);
  } else {
#pragma unroll
    for (int k = 0; k < kC; ++k)
      if (e + k < n) p[e + k] = r.v[k];
  }
}

// ---- reduction bodies / finalisers (pCG) ----
struct CgInitBody {  // sums p.p and r.z  (z == p initially)
  const double *p, *r;
  int64_t n;
  __device__ void setup() {}
  __device__ void operator()(int64_t c, double (&a)[2]) const {
    const V4 pv = ld4(p, c * kC, n), rv = ld4(r, c * kC, n);
#pragma unroll
    for (int k = 0; k < kC; ++k) {
      a[0] = fma(pv.v[k], pv.v[k], a[0]);
      a[1] = fma(rv.v[k], pv.v[k], a[1]);
    }
  }
};
struct CgInitFin {
  KHead* head;
  double tol;
  double* hist;
  __device__ void operator()(const double (&s)[2]) const {
    const double res0 = sqrt(s[0]);  // res_mag[0] = sqrt(dot(p, p))
    head->res0 = res0;
    head->res = res0;
    head->tolerance = res0 * tol;
    head->rz = s[1];
    head->j = 0;
    hist[0] = res0;
    head->n_hist = 1;
    head->done = (res0 > head->tolerance) ? DONE_RUNNING : DONE_CONVERGED;
    if (!isfinite(res0)) head->done = DONE_NAN;
  }
};
struct CgPApBody {
  const double *p, *Ap;
  int64_t n;
  __device__ void setup() {}
  __device__ void operator()(int64_t c, double (&a)[1]) const {
    const V4 pv = ld4(p, c * kC, n), av = ld4(Ap, c * kC, n);
#pragma unroll
    for (int k = 0; k < kC; ++k) a[0] = fma(pv.v[k], av.v[k], a[0]);
  }
};
struct CgPApFin {
  KHead* head;
  __device__ void operator()(const double (&s)[1]) const {
    head->pAp = s[0];
    head->alpha = head->rz / s[0];  // alpha = rz / dot(p, Ap)
  }
};
struct CgUpdBody {  // x += alpha p; r -= alpha Ap; sum r.r
  double *x, *r;
  const double *p, *Ap;
  const KHead* head;
  double alpha;
  int64_t n;
  __device__ void setup() { alpha = head->alpha; }
  __device__ void operator()(int64_t c, double (&a)[1]) {
    const int64_t e = c * kC;
    V4 xv = ld4(x, e, n), rv = ld4(r, e, n);
    const V4 pv = ld4(p, e, n), av = ld4(Ap, e, n);
#pragma unroll
    for (int k = 0; k < kC; ++k) {
      xv.v[k] += alpha * pv.v[k];
      rv.v[k] = rv.v[k] - alpha * av.v[k];
      a[0] = fma(rv.v[k], rv.v[k], a[0]);
    }
    st4(x, e, n, xv);
    st4(r, e, n, rv);
  }
};
struct CgUpdFin {
  KHead* head;
  double* hist;
  int hist_cap;
  __device__ void operator()(const double (&s)[1]) const {
    const double res = sqrt(s[0]);
    head->res = res;
    if (head->n_hist < hist_cap) hist[head->n_hist] = res;
    head->n_hist++;
    if (!isfinite(res) || !isfinite(head->alpha)) head->done = DONE_NAN;
    else if (!(res > head->tolerance)) head->done = DONE_CONVERGED;
  }
};
struct CgRzBody {
  const double *r, *z;
  int64_t n;
  __device__ void setup() {}
  __device__ void operator()(int64_t c, double (&a)[1]) const {
    const V4 rv = ld4(r, c * kC, n), zv = ld4(z, c * kC, n);
#pragma unroll
    for (int k = 0; k < kC; ++k) a[0] = fma(rv.v[k], zv.v[k], a[0]);
  }
};
struct CgRzFin {
  KHead* head;
  int max_iters;
  __device__ void operator()(const double (&s)[1]) const {
    head->beta = s[0] / head->rz;  // beta = dot(r, z) / rz
    head->rz = s[0];
    head->j++;
    if (head->j > max_iters) head->done = DONE_MAXIT;
  }
};

// ---- reduction bodies (pGMRES) ----
struct NormFin {  // ||v|| into *out
  double* out;
  __device__ void operator()(const double (&s)[1]) const { *out = sqrt(fabs(s[0])); }
};
// pass i of MGS for column j: v -= H(i-1, j) q_{i-1} (i > 0); H(i, j) = q_i . v
struct MgsBody {
  double* v;
  const double *qprev, *qi;
  const double* hprev_ptr;
  double hprev;
  int64_t n;
  __device__ void setup() { hprev = qprev ? *hprev_ptr : 0.0; }
  __device__ void operator()(int64_t c, double (&a)[1]) {
    const int64_t e = c * kC;
    V4 vv = ld4(v, e, n);
    const V4 qv = ld4(qi, e, n);
    if (qprev) {
      const V4 pv = ld4(qprev, e, n);
#pragma unroll
      for (int k = 0; k < kC; ++k) vv.v[k] = fma(-hprev, pv.v[k], vv.v[k]);
      st4(v, e, n, vv);
    }
#pragma unroll
    for (int k = 0; k < kC; ++k) a[0] = fma(qv.v[k], vv.v[k], a[0]);
  }
};
// last pass: v -= H(j, j) q_j; H(j+1, j) = ||v||
struct MgsLastBody {
  double* v;
  const double* qj;
  const double* h_ptr;
  double h;
  int64_t n;
  __device__ void setup() { h = *h_ptr; }
  __device__ void operator()(int64_t c, double (&a)[1]) {
    const int64_t e = c * kC;
    V4 vv = ld4(v, e, n);
    const V4 qv = ld4(qj, e, n);
#pragma unroll
    for (int k = 0; k < kC; ++k) {
      vv.v[k] = fma(-h, qv.v[k], vv.v[k]);
      a[0] = fma(vv.v[k], vv.v[k], a[0]);
    }
    st4(v, e, n, vv);
  }
};

// ---- modified Gram-Schmidt of one Arnoldi column in one persistent launch
// (one_arnoldi, blocksp_solvers.hpp:109-136):
//   for i = 0..j: H(i, j) = q_i . v;  v -= H(i, j) q_i
//   H(j+1, j) = ||v||;  q_{j+1} = v / H(j+1, j) (unless below zero_thresh)
// One CTA per SM, all co-resident (cooperative launch).  Each CTA keeps its
// slice of v in registers for the whole column and the slice of the last
// basis vector in shared memory, so a pass reads one basis vector from HBM
// (the per-pass launch form reads v and q_{i-1}, q_i and writes v back).
// Passes are separated by a bounded grid barrier; every CTA sums the per-CTA
// partials in index order, so H is bit-reproducible.  The update and the dot
// use the same fma sequence as the per-pass form, in MGS order.
constexpr int kMgsThreads = 1024;

struct MgsP {
  int64_t len;
  int64_t slice;           // elements per CTA
  const double* v;         // M^-1 A q_j
  double* const* Q;        // basis table
  int j;                   // column
  double* H;               // (m+1) x m, row-major, leading dimension ldh
  int ldh;
  const KHead* head;       // zero_thresh
  double* partials;        // (j+2) x gridDim.x
  unsigned* bar;           // barrier counter (0 at launch)
  unsigned spin_limit;
  DevStatus* st;
};

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Sum over the CTA (every thread gets the result).
__device__ __forceinline__ double cta_sum_1024(double a, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
  if (lane == 0) red[warp] = a;
  __syncthreads();
  if (warp == 0) {
    double t = red[lane];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (lane == 0) red[32] = t;
  }
  __syncthreads();
  const double r = red[32];
  __syncthreads();
  return r;
}

// Grid barrier number `gen` (1, 2, ...): bounded spin, BSP_TIMEOUT on expiry.
__device__ __forceinline__ void mgs_barrier(const MgsP& p, unsigned gen) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(p.bar, 1u);
    const unsigned target = gen * gridDim.x;
    unsigned spins = 0;
    while (ld_acquire_u32(p.bar) < target) {
      if (++spins > p.spin_limit) {
        set_status(p.st, BSP_TIMEOUT, -1);
        break;
      }
      poll_pause(spins);
    }
    __threadfence();
  }
  __syncthreads();
}

// Asks L2 to fetch n doubles at src (a hint: nothing is written; a range
// that is not 16-byte aligned is skipped).  Called by warp 0 of the CTA:
// lane k issues the k-th 16 KB piece.
__device__ __forceinline__ void prefetch_l2(const double* src, int64_t n) {
  const uintptr_t a = reinterpret_cast<uintptr_t>(src);
  if (n <= 0 || (a & 15u)) return;
  const int64_t bytes = (n * 8) & ~int64_t(15);
  constexpr int64_t kPiece = 16384;
  for (int64_t o = (int64_t)(threadIdx.x & 31) * kPiece; o < bytes; o += 32 * kPiece) {
    const unsigned sz = (unsigned)(bytes - o < kPiece ? bytes - o : kPiece);
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a + o), "r"(sz) : "memory");
  }
}

// Sum of the gridDim.x partials of one pass, in index order (same in every CTA).
__device__ __forceinline__ double grid_total(const double* part, double* red) {
  if (threadIdx.x < 32) {
    double a = 0.0;
    for (int c = threadIdx.x; c < (int)gridDim.x; c += 32) a += __ldcg(part + c);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (threadIdx.x == 0) red[33] = a;
  }
  __syncthreads();
  const double r = red[33];
  __syncthreads();
  return r;
}

template <int NPT>
__global__ void __launch_bounds__(kMgsThreads, 1) k_mgs(const MgsP p) {
  extern __shared__ double qs[];  // this CTA's slice of the last basis vector
  __shared__ double red[34];
  const int t = threadIdx.x;
  const int64_t beg = (int64_t)blockIdx.x * p.slice;
  const int nloc = (int)((beg + p.slice < p.len ? beg + p.slice : p.len) - beg);  // may be <= 0
  // the first two basis vectors' slices start streaming into L2 now; later
  // ones two passes ahead of their use
  if (t < 32) {
    prefetch_l2(p.Q[0] + beg, nloc);
    if (p.j >= 1) prefetch_l2(p.Q[1] + beg, nloc);
  }
  double v[NPT];
  {
    const double* vb = p.v + beg;
#pragma unroll
    for (int k = 0; k < NPT; ++k) {
      const int o = t + k * kMgsThreads;
      v[k] = o < nloc ? vb[o] : 0.0;
    }
  }
  double h = 0.0;
  unsigned gen = 0;
  for (int i = 0; i <= p.j; ++i) {
    const double* qb = p.Q[i] + beg;
    double a = 0.0;
    // the axpy with the previous basis vector (its slice in shared memory),
    // then this vector's slice replaces it: one batch of copies in flight at
    // once (each thread copies and reads only its own entries)
    if (i > 0) {
#pragma unroll
      for (int k = 0; k < NPT; ++k) {
        const int o = t + k * kMgsThreads;
        if (o < nloc) v[k] = fma(-h, qs[o], v[k]);
      }
    }
#pragma unroll
    for (int k = 0; k < NPT; ++k) {
      const int o = t + k * kMgsThreads;
      if (o < nloc) cp_async_small<8>(qs + o, qb + o);
    }
    cp_async_commit();
    cp_async_wait<0>();
#pragma unroll
    for (int k = 0; k < NPT; ++k) {
      const int o = t + k * kMgsThreads;
      if (o < nloc) a = fma(qs[o], v[k], a);
    }
    a = cta_sum_1024(a, red);
    if (t == 0) p.partials[(size_t)i * gridDim.x + blockIdx.x] = a;
    // a later basis vector's slice streams into L2 while the grid meets
    if (t < 32 && i + 2 <= p.j) prefetch_l2(p.Q[i + 2] + beg, nloc);
    mgs_barrier(p, ++gen);
    h = grid_total(p.partials + (size_t)i * gridDim.x, red);
    if (blockIdx.x == 0 && t == 0) p.H[(size_t)i * p.ldh + p.j] = h;
  }
  double a = 0.0;
#pragma unroll
  for (int k = 0; k < NPT; ++k) {
    const int o = t + k * kMgsThreads;
    if (o < nloc) {
      v[k] = fma(-h, qs[o], v[k]);
      a = fma(v[k], v[k], a);
    }
  }
  a = cta_sum_1024(a, red);
  if (t == 0) p.partials[(size_t)(p.j + 1) * gridDim.x + blockIdx.x] = a;
  mgs_barrier(p, ++gen);
  const double nrm = sqrt(fabs(grid_total(p.partials + (size_t)(p.j + 1) * gridDim.x, red)));
  if (blockIdx.x == 0 && t == 0) p.H[(size_t)(p.j + 1) * p.ldh + p.j] = nrm;
  if (fabs(nrm) < p.head->zero_thresh) return;  // breakdown: the basis is not extended
  double* qn = p.Q[p.j + 1] + beg;
#pragma unroll
  for (int k = 0; k < NPT; ++k) {
    const int o = t + k * kMgsThreads;
    if (o < nloc) qn[o] = v[k] / nrm;
  }
}

struct GPtrs {
  KHead* head;
  int m;  // leading dimension / capacity in columns
  double *H, *R, *g, *rhs, *y;
  sd::Rot* rots;
  int* nrot;
  double* hist;
  int hist_cap;
  // deflated restart work
  double *Hn, *Z, *P, *w, *work, *wr, *wi, *resv, *Hnew;
  int *perm, *sel;
};

__global__ void k_gm_init(GPtrs g, double tol) {
  KHead* h = g.head;
  const double res0 = h->res0;  // written by the norm reduction
  h->res = res0;
  h->tolerance = res0 * tol;
  h->zero_thresh = fmin(res0 * kEps, kEps);
  h->j = 0;
  h->tot = 0;
  h->restarted = 0;
  h->breakdown = 0;
  h->keff = 0;
  g.hist[0] = res0;
  h->n_hist = 1;
  for (int i = 0; i <= g.m; ++i) {
    g.g[i] = 0.0;
    g.rhs[i] = 0.0;
  }
  g.g[0] = res0;
  g.rhs[0] = res0;
  *g.nrot = 0;
  h->done = (res0 > h->tolerance) ? DONE_RUNNING : DONE_CONVERGED;
  if (!isfinite(res0)) h->done = DONE_NAN;
}

// Least-squares update after column j was built (H(0..j+1, j) in place).
__global__ void k_gm_ls(GPtrs g, int max_iters) {
  KHead* h = g.head;
  const int j = h->j;
  const double hsub = g.H[(j + 1) * g.m + j];
  if (fabs(hsub) < h->zero_thresh) h->breakdown = 1;
  int nrot = *g.nrot;
  const double res = sd::ls_add_column(g.H, g.m, j, j + 1, g.R, g.rots, nrot, g.g);
  *g.nrot = nrot;
  h->res = res;
  if (h->n_hist < g.hist_cap) g.hist[h->n_hist] = res;
  h->n_hist++;
  h->j = j + 1;
  h->tot++;
  if (!isfinite(res)) h->done = DONE_NAN;
  else if (!(res > h->tolerance)) h->done = DONE_CONVERGED;
  else if (h->tot > max_iters) h->done = DONE_MAXIT;
  else if (h->breakdown) h->done = DONE_BREAKDOWN;
}

// y = R^{-1} g over the current n = j columns
__global__ void k_gm_y(GPtrs g) { sd::back_solve(g.R, g.m, g.g, g.head->j, g.y); }

// x += sum_i y_i q_i  (in the reference's order: x = x0 + y0 q0 + y1 q1 + ...)
__global__ void k_gm_combine(int64_t len, double* __restrict__ x, double* const* __restrict__ Q,
                             const double* __restrict__ y, const KHead* __restrict__ head) {
  const int n = head->j;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < len; e += (int64_t)gridDim.x * blockDim.x) {
    double xe = x[e];
    for (int i = 0; i < n; ++i) xe += y[i] * Q[i][e];
    x[e] = xe;
  }
}

// Shared-memory footprint (doubles, then ints) of the deflated restart's
// working set for restart length m; the kernel stages it in shared memory
// when it fits and otherwise works in the global scratch.
inline size_t deflate_smem_bytes(int m) {
  const size_t d = (size_t)m * m * 2 + ((size_t)m * m + 4 * (size_t)m + 32) + (size_t)(m + 1) * (m + 2) +
                   3 * (size_t)(m + 1) + (size_t)(m + 2);
  return d * sizeof(double) + 2 * (size_t)m * sizeof(int);
}
constexpr size_t kDeflateSmemMax = 200 * 1024;

// Deflated restart (deflated_restart.hpp:38-269) on one warp.
// Input: H ((n+1) x n, n = head->j), rhs, y (current LS solution), k.
// Output: P_{k+1} in g.P ((n+1) x (keff+1), ld = m+1), H_new, c_r, new LS state.
__global__ void __launch_bounds__(32) k_gm_deflate(GPtrs g, int k_req, int max_keep, int use_smem) {
  extern __shared__ __align__(16) double dsm[];
  const sd::WarpTeam tm;
  const int r0 = tm.rank(), ns = tm.size();
  KHead* h = g.head;
  const int n = h->j, m1 = n + 1, ld = g.m;
  int k = k_req > n ? n : k_req;
  // working arrays: shared memory when they fit, else the global scratch
  GPtrs L = g;
  if (use_smem) {
    double* b = dsm;
    const int m = g.m;
    L.Hn = b; b += (size_t)m * m;
    L.Z = b; b += (size_t)m * m;
    L.work = b; b += (size_t)m * m + 4 * (size_t)m + 32;
    L.P = b; b += (size_t)(m + 1) * (m + 2);
    L.w = b; b += m + 1;
    L.wr = b; b += m + 1;
    L.wi = b; b += m + 1;
    L.resv = b; b += m + 2;
    L.perm = reinterpret_cast<int*>(b);
    L.sel = L.perm + m;
  }
  // residual vector res_vec = rhs - H y (solvers.hpp:202-203, 226-227)
  for (int i = r0; i < m1; i += ns) {
    double s = 0.0;
    for (int t = 0; t < n; ++t) s += g.H[i * ld + t] * g.y[t];
    L.resv[i] = g.rhs[i] - s;
  }
  const double zero_thresh = 10.0 * n * n * kEps;
  // (1) H_tilde = H_n + |h_mn|^2 H_n^{-T} e_n e_n^T
  const int ldn = g.m;
  for (int e = r0; e < n * n; e += ns) {
    const int i = e / n, t = e % n;
    L.Hn[i * ldn + t] = g.H[i * ld + t];
  }
  const double hmn = g.H[n * ld + n - 1];
  for (int i = r0; i < n; i += ns) L.w[i] = (i == n - 1) ? 1.0 : 0.0;
  tm.sync();
  sd::solve_transposed(tm, L.Hn, ldn, n, L.w, L.work, L.perm);
  for (int i = r0; i < n; i += ns) L.Hn[i * ldn + n - 1] += hmn * hmn * L.w[i];
  tm.sync();
  // (2) real Schur form, selection of the k smallest harmonic Ritz values
  sd::hessenberg(tm, L.Hn, ldn, n, L.Z, ldn, L.work);
  const bool conv = sd::francis_qr(tm, L.Hn, ldn, n, L.Z, ldn);
  if (r0 == 0) {
    sd::schur_eigs(L.Hn, ldn, n, L.wr, L.wi);
    sd::select_smallest(L.wr, L.wi, n, k, zero_thresh, L.perm, L.sel);
  }
  tm.sync();
  // (3) orthonormal basis P_k of the selected invariant subspace
  const int ldp = g.m + 1;
  const int keff = sd::invariant_basis(tm, L.Hn, ldn, n, L.Z, ldn, L.wr, L.wi, L.sel, L.P, ldp, L.work);
  k = keff;
  if (!conv || k < 1 || k + 1 > max_keep) {
    if (r0 == 0) {
      h->done = DONE_BREAKDOWN;  // the Qn update below is skipped (keff = -1)
      h->keff = -1;
    }
    return;
  }
  // (4) P_{k+1}: [P_k; 0] and res_vec orthogonalised (classical GS as in :211-232)
  for (int t = r0; t < k; t += ns) L.P[n * ldp + t] = 0.0;
  for (int i = r0; i < m1; i += ns) L.P[i * ldp + k] = L.resv[i];
  tm.sync();
  for (int c = 0; c < k; ++c) {
    double d = 0.0;
    for (int i = r0; i < m1; i += ns) d += L.P[i * ldp + c] * L.P[i * ldp + k];
    d = tm.sum(d);
    for (int i = r0; i < m1; i += ns) L.P[i * ldp + k] -= d * L.P[i * ldp + c];
    tm.sync();
  }
  {
    double nrm = 0.0;
    for (int i = r0; i < m1; i += ns) nrm += L.P[i * ldp + k] * L.P[i * ldp + k];
    nrm = sqrt(tm.sum(nrm));
    for (int i = r0; i < m1; i += ns) L.P[i * ldp + k] /= nrm;
    tm.sync();
  }
  // (5) c_r = P_{k+1}^T res_vec
  for (int c = r0; c <= k; c += ns) {
    double s = 0.0;
    for (int i = 0; i < m1; ++i) s += L.P[i * ldp + c] * L.resv[i];
    g.rhs[c] = s;
  }
  for (int i = k + 1 + r0; i <= g.m; i += ns) g.rhs[i] = 0.0;
  // (6) H_new = P_{k+1}^T H P_k  ((k+1) x k); W = H P_k in g.Hnew ((n+1) x k, ld = m)
  for (int e = r0; e < m1 * k; e += ns) {
    const int i = e / k, c = e % k;
    double s = 0.0;
    for (int t = 0; t < n; ++t) s += g.H[i * ld + t] * L.P[t * ldp + c];
    g.Hnew[i * ld + c] = s;
  }
  tm.sync();
  for (int e = r0; e < (k + 1) * k; e += ns) {
    const int r = e / k, c = e % k;
    double s = 0.0;
    for (int i = 0; i < m1; ++i) s += L.P[i * ldp + r] * g.Hnew[i * ld + c];
    L.work[r * ld + c] = s;
  }
  tm.sync();
  for (int e = r0; e < (g.m + 1) * g.m; e += ns) {
    const int r = e / g.m, c = e % g.m;
    g.H[e] = (r <= k && c < k) ? L.work[r * ld + c] : 0.0;
  }
  // P_{k+1} to the global scratch for the Qn update
  if (use_smem)
    for (int e = r0; e < m1 * (k + 1); e += ns) {
      const int i = e / (k + 1), c = e % (k + 1);
      g.P[i * ldp + c] = L.P[i * ldp + c];
    }
  tm.sync();
  // (8) restart the least-squares state from H_new and c_r
  if (r0 == 0) {
    int nrot = 0;
    for (int i = 0; i <= g.m; ++i) g.g[i] = g.rhs[i];
    for (int c = 0; c < k; ++c) sd::ls_add_column(g.H, ld, c, k, g.R, g.rots, nrot, g.g);
    *g.nrot = nrot;
    h->keff = k;
    h->j = k;
    h->restarted = 1;
  }
}

// Qout[0..k] <- Qn[0..m1-1] P_{k+1} (deflated_restart.hpp:250-258), written to
// spare vectors; the host then swaps the pointer tables.
// Qout[c] = sum_i Q[i] P[i][c] for c <= keff: each thread reads its entry of
// the m1 basis vectors once (in chunks of 32, in registers) and forms every
// output column from them, summing in basis order; P sits in shared memory.
// Up to kQnCols output columns; wider restarts take the column-by-column loop.
constexpr int kQnCols = 16;
__global__ void __launch_bounds__(256) k_gm_qn_update(int64_t len, double* const* __restrict__ Q,
                                                      double* const* __restrict__ Qout, const double* __restrict__ P,
                                                      int ldp, const KHead* __restrict__ head, int m1) {
  extern __shared__ double ps[];  // m1 x kQnCols
  const int kp1 = head->keff + 1;  // <= the spare count, checked by k_gm_deflate
  if (kp1 > kQnCols) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < len; e += (int64_t)gridDim.x * blockDim.x) {
      for (int c = 0; c < kp1; ++c) {
        double s = 0.0;
        for (int i = 0; i < m1; ++i) s += Q[i][e] * P[i * ldp + c];
        Qout[c][e] = s;
      }
    }
    return;
  }
  for (int t = threadIdx.x; t < m1 * kQnCols; t += blockDim.x) {
    const int i = t / kQnCols, c = t % kQnCols;
    ps[t] = c < kp1 ? P[i * ldp + c] : 0.0;
  }
  __syncthreads();
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < len; e += (int64_t)gridDim.x * blockDim.x) {
    double s[kQnCols];
#pragma unroll
    for (int c = 0; c < kQnCols; ++c) s[c] = 0.0;
    for (int i0 = 0; i0 < m1; i0 += 32) {
      double qv[32];
#pragma unroll
      for (int t = 0; t < 32; ++t) qv[t] = i0 + t < m1 ? __ldcs(Q[i0 + t] + e) : 0.0;
#pragma unroll
      for (int t = 0; t < 32; ++t)
        if (i0 + t < m1) {
#pragma unroll
          for (int c = 0; c < kQnCols; ++c) s[c] += qv[t] * ps[(i0 + t) * kQnCols + c];
        }
    }
#pragma unroll
    for (int c = 0; c < kQnCols; ++c)
      if (c < kp1) Qout[c][e] = s[c];
  }
}

// Pure restart (k = 0): q_0 = r_0 / ||r_0||, rhs = ||r_0|| e_1 (solvers.hpp:255-262)
__global__ void k_gm_pure_restart(GPtrs g) {
  KHead* h = g.head;
  const double r = h->res0;  // holds ||r_0|| of the new residual here
  if (h->n_hist < g.hist_cap) g.hist[h->n_hist] = r;
  h->n_hist++;
  for (int i = 0; i <= g.m; ++i) {
    g.g[i] = 0.0;
    g.rhs[i] = 0.0;
  }
  g.g[0] = r;
  g.rhs[0] = r;
  *g.nrot = 0;
  h->j = 0;
  h->keff = 0;
  h->restarted = 0;
  h->res = r;
  if (!(r > h->tolerance)) h->done = DONE_CONVERGED;
}

// Eigenvalues of the square part H_s (n x n) of H ((n+1) x n, leading
// dimension ldh), or harmonic Ritz values when harmonic (Eigenvalues_Arr,
// blocksp_dense_solvers.hpp:916-961): one warp, scratch in global memory.
__global__ void __launch_bounds__(32) k_ritz(const double* __restrict__ H, int ldh, int n, int harmonic,
                                             double* work, int* iwork, double* wr, double* wi, int* ok) {
  const sd::WarpTeam tm;
  const int r0 = tm.rank(), ns = tm.size();
  double* Hn = work;
  double* Z = Hn + (size_t)n * n;
  double* scr = Z + (size_t)n * n;
  double* w = scr + (size_t)n * n + 4 * (size_t)n + 32;
  for (int e = r0; e < n * n; e += ns) Hn[e] = H[(size_t)(e / n) * ldh + e % n];
  tm.sync();
  if (harmonic) {
    // H_tilde = H_n + h_mn^2 H_n^-T e_n e_n^T (only the last column changes)
    const double hmn = H[(size_t)n * ldh + n - 1];
    for (int i = r0; i < n; i += ns) w[i] = (i == n - 1) ? 1.0 : 0.0;
    tm.sync();
    sd::solve_transposed(tm, Hn, n, n, w, scr, iwork);
    for (int i = r0; i < n; i += ns) Hn[(size_t)i * n + n - 1] += hmn * hmn * w[i];
    tm.sync();
  }
  sd::hessenberg(tm, Hn, n, n, Z, n, scr);
  const bool conv = sd::francis_qr(tm, Hn, n, n, Z, n);
  if (r0 == 0) {
    sd::schur_eigs(Hn, n, n, wr, wi);
    *ok = conv ? 1 : 0;
  }
}

// printEigInfo / printEigVals text of Eigenvalues_Arr (dense_solvers.hpp:973-990).
void print_eigs(const double* wr, const double* wi, int n, bool harmonic, bool info, bool vals) {
  if (n < 1) return;
  std::vector<double> wm(n);
  for (int i = 0; i < n; ++i) wm[i] = std::sqrt(wr[i] * wr[i] + wi[i] * wi[i]);
  auto mn = [&](const double* a) { return *std::min_element(a, a + n); };
  auto mx = [&](const double* a) { return *std::max_element(a, a + n); };
  if (vals) {
    if (harmonic) printf("Harmonic Ritz values\n");
    printf("Eigenvalues - real component\n");
    for (int i = 0; i < n; ++i) printf("%g%c", wr[i], i + 1 < n ? ' ' : '\n');
    printf("Eigenvalues - imaginary component\n");
    for (int i = 0; i < n; ++i) printf("%g%c", wi[i], i + 1 < n ? ' ' : '\n');
    printf("Eigenvalues - magnitude\n");
    for (int i = 0; i < n; ++i) printf("%g%c", wm[i], i + 1 < n ? ' ' : '\n');
  }
  if (info) {
    printf(harmonic ? "Harmonic Ritz info\n" : "Eigenvalue info\n");
    printf("min/max real eig %g %g\n", mn(wr), mx(wr));
    printf("min/max img  eig %g %g\n", mn(wi), mx(wi));
    printf("smallest magn eig %g\n", mn(wm.data()));
    printf("largest magn eig  %g\n", mx(wm.data()));
    printf("ratio/cond %g\n", mx(wm.data()) / mn(wm.data()));
  }
  fflush(stdout);
}

// Ritz values of the n-column H (device, leading dimension ldh) to the host.
static int ritz_values(bsp_handle_s* h, const double* H, int ldh, int n, bool harmonic, double* wr, double* wi) {
  if (n < 1) return BSP_OK;
  double* work = nullptr;
  int* iwork = nullptr;
  BSP_TRY(h->scratch("ritz.work", (size_t)3 * n * n + 7 * (size_t)n + 64, &work));
  BSP_TRY(h->scratch("ritz.iwork", (size_t)n + 1, &iwork));
  double* wdev = work + (size_t)3 * n * n + 5 * (size_t)n + 32;  // 2n values
  bsp::count_launch(), k_ritz<<<1, 32, 0, h->stream>>>(H, ldh, n, harmonic ? 1 : 0, work, iwork + 1, wdev,
                                                       wdev + n, iwork);
  BSP_CUDA_TRY(cudaPeekAtLastError());
  std::vector<double> wv(2 * (size_t)n);
  int ok = 0;
  BSP_CUDA_TRY(cudaMemcpyAsync(wv.data(), wdev, 2 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  BSP_CUDA_TRY(cudaMemcpyAsync(&ok, iwork, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  BSP_CUDA_TRY(cudaStreamSynchronize(h->stream));
  if (!ok) {
    record_error("eigenvalues: the QR iteration did not converge");
    return BSP_BREAKDOWN;
  }
  std::copy(wv.begin(), wv.begin() + n, wr);
  std::copy(wv.begin() + n, wv.end(), wi);
  return BSP_OK;
}

// ------------------------------------------------------------------ host helpers
// One persistent MGS launch for column j when the slice of v fits the
// registers of one CTA per SM (else returns 1: the per-pass form is used).
template <int NPT>
static int launch_mgs_t(bsp_handle_s* h, MgsP& p, int grid) {
  const size_t smem = (size_t)NPT * kMgsThreads * sizeof(double);
  static bool ok = false;
  if (!ok) {
    BSP_CUDA_TRY(cudaFuncSetAttribute(k_mgs<NPT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    BSP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_mgs<NPT>, kMgsThreads, smem));
    if (per_sm < 1) return 1;
    ok = true;
  }
  void* args[] = {&p};
  bsp::count_launch();
  BSP_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)k_mgs<NPT>, grid, kMgsThreads, args, smem, h->stream));
  return BSP_OK;
}

static int launch_mgs(bsp_handle_s* h, int64_t len, const double* v, double* const* Q, int j, double* H, int ldh,
                      const KHead* head, double* partials, unsigned* bar) {
  const int grid = h->num_sms;
  const int64_t per_thread = (len + (int64_t)grid * kMgsThreads - 1) / ((int64_t)grid * kMgsThreads);
  MgsP p{};
  p.len = len;
  p.v = v;
  p.Q = Q;
  p.j = j;
  p.H = H;
  p.ldh = ldh;
  p.head = head;
  p.partials = partials;
  p.bar = bar;
  p.spin_limit = h->spin_limit;
  p.st = h->ws.status.get();
  BSP_CUDA_TRY(cudaMemsetAsync(bar, 0, sizeof(unsigned), h->stream));
  auto run = [&](auto npt) -> int {
    constexpr int N = decltype(npt)::value;
    p.slice = (int64_t)N * kMgsThreads;
    if (p.slice * grid < len) return 1;
    return launch_mgs_t<N>(h, p, grid);
  };
  if (per_thread <= 4) return run(std::integral_constant<int, 4>{});
  if (per_thread <= 8) return run(std::integral_constant<int, 8>{});
  if (per_thread <= 16) return run(std::integral_constant<int, 16>{});
  if (per_thread <= 24) return run(std::integral_constant<int, 24>{});
  return 1;
}

static int read_head(bsp_handle_s* h, const KHead* d, KHead* out) {
  BSP_CUDA_TRY(cudaMemcpyAsync(out, d, sizeof(KHead), cudaMemcpyDeviceToHost, h->stream));
  BSP_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return BSP_OK;
}

static int status_of(int done) {
  switch (done) {
    case DONE_CONVERGED: return BSP_OK;
    case DONE_MAXIT: return BSP_MAXIT;
    case DONE_BREAKDOWN: return BSP_BREAKDOWN;
    case DONE_NAN: return BSP_NAN;
    default: return BSP_OK;
  }
}

int true_residual(bsp_handle_s* h, bsp_matrix_s* A, const double* b, const double* x, double* work,
                  double* out_host) {
  const int64_t len = (int64_t)A->n_rows * A->bs;
  BSP_TRY(bsmv_launch(A, 1, 0, BSP_F64, -1.0, x, 1.0, b, work, h->stream));
  double* s = h->ws.scalars.get();
  BSP_TRY(launch_reduce<1>(h, 1, len, DotBody{work, work}, StoreFin{s}));
  BSP_TRY(launch_reduce<1>(h, 2, len, DotBody{b, b}, StoreFin{s + 1}));
  double v[2];
  BSP_CUDA_TRY(cudaMemcpyAsync(v, s, 2 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  BSP_CUDA_TRY(cudaStreamSynchronize(h->stream));
  *out_host = v[1] > 0 ? sqrt(v[0]) / sqrt(v[1]) : sqrt(v[0]);
  return BSP_OK;
}


// ------------------------------------------------------------------ pCG
// Stored copy of A the inner operator reads: FP64 for the reference method,
// FP32 or BF16 storage (FP64 vectors and accumulation) for the mixed modes.
static int op_dtype_of(int op_prec) {
  return op_prec == BSP_PREC_F64 ? BSP_F64 : op_prec == BSP_PREC_F32 ? BSP_F32_STORE : BSP_BF16_STORE;
}

int pcg_solve(bsp_handle_s* h, bsp_matrix_s* A, bsp_precond_s* pc, const double* b, double* x,
              const bsp_solve_opts* o, double* hist, int hist_cap, bsp_solve_info* info,
              int op_prec = BSP_PREC_F64, bool want_true = true) {
  const int op_dtype = op_dtype_of(op_prec);
  const int64_t len = (int64_t)A->n_rows * A->bs;
  const int hcap = std::max(2, o->max_iters + 3);
  Span<double> vr, vp, vz, vAp, dhist;
  Span<KHead> dhead;
  BSP_TRY(h->scratch("pcg.r", len, &vr.p));
  BSP_TRY(h->scratch("pcg.p", len, &vp.p));
  BSP_TRY(h->scratch("pcg.z", len, &vz.p));
  BSP_TRY(h->scratch("pcg.Ap", len, &vAp.p));
  BSP_TRY(h->scratch("pcg.hist", hcap, &dhist.p));
  BSP_TRY(h->scratch("pcg.head", 1, &dhead.p));
  BSP_CUDA_TRY(cudaMemsetAsync(dhead.get(), 0, sizeof(KHead), h->stream));
  EventTimer tm(h->stream);
  const int g = grid_for(h, len, 256);
  KHead* hd = dhead.get();
  BSP_CUDA_TRY(cudaMemsetAsync(x, 0, len * sizeof(double), h->stream));      // x = 0
  bsp::count_launch(), k_copy<<<g, 256, 0, h->stream>>>(len, b, vr.get());                         // r = b
  if (pc) BSP_TRY(precond_apply(pc, op_prec,b, vp.get()));              // p = M^-1 b
  else bsp::count_launch(), k_copy<<<g, 256, 0, h->stream>>>(len, b, vp.get());
  bsp::count_launch(), k_copy<<<g, 256, 0, h->stream>>>(len, vp.get(), vz.get());                  // z = p
  BSP_TRY(launch_reduce<2>(h, 3, chunks_of(len), CgInitBody{vp.get(), vr.get(), len}, CgInitFin{hd, o->tol, dhist.get()}));
  KHead st;
  BSP_TRY(read_head(h, hd, &st));
  while (st.done == DONE_RUNNING) {
    BSP_TRY(bsmv_launch(A, 1, 0, op_dtype, 1.0,vp.get(), 0.0, nullptr, vAp.get(), h->stream));
    BSP_TRY(launch_reduce<1>(h, 4, chunks_of(len), CgPApBody{vp.get(), vAp.get(), len}, CgPApFin{hd}));
    BSP_TRY(launch_reduce<1>(h, 5, chunks_of(len), CgUpdBody{x, vr.get(), vp.get(), vAp.get(), hd, 0.0, len},
                             CgUpdFin{hd, dhist.get(), hcap}));
    BSP_TRY(read_head(h, hd, &st));
    if (st.done != DONE_RUNNING) break;
    if (pc) BSP_TRY(precond_apply(pc, op_prec,vr.get(), vz.get()));
    else bsp::count_launch(), k_copy<<<g, 256, 0, h->stream>>>(len, vr.get(), vz.get());
    BSP_TRY(launch_reduce<1>(h, 6, chunks_of(len), CgRzBody{vr.get(), vz.get(), len}, CgRzFin{hd, o->max_iters}));
    bsp::count_launch(), k_cg_p<<<g, 256, 0, h->stream>>>(len, vz.get(), hd, vp.get());
    BSP_CUDA_TRY(cudaPeekAtLastError());
    BSP_TRY(read_head(h, hd, &st));
  }
  const double solve_ms = tm.stop_ms();
  if (pc) BSP_TRY(precond_check_status(pc));
  const int nh = std::min(st.n_hist, hcap);
  if (hist && hist_cap > 0)
    BSP_CUDA_TRY(cudaMemcpy(hist, dhist.get(), std::min(nh, hist_cap) * sizeof(double), cudaMemcpyDeviceToHost));
  if (info) {
    info->status = status_of(st.done);
    info->iters = st.j;
    info->n_hist = nh;
    info->n_restarts = 0;
    info->res0 = st.res0;
    info->final_res = st.res;
    info->solve_ms = solve_ms;
    if (want_true) BSP_TRY(true_residual(h, A, b, x, vAp.get(), &info->true_rel_res));
  }
  if (o->print_iters) {
    printf("pCG iters %d\n", st.j);  // solvers.hpp:99-103
    if (st.j > o->max_iters) printf("maximum pCG iterations reached\n");
  }
  return status_of(st.done);
}

// ------------------------------------------------------------------ pGMRES
int pgmres_solve(bsp_handle_s* h, bsp_matrix_s* A, bsp_precond_s* pc, const double* b, double* x,
                 const bsp_solve_opts* o, double* hist, int hist_cap, bsp_solve_info* info,
                 int op_prec = BSP_PREC_F64, bool want_true = true) {
  const int op_dtype = op_dtype_of(op_prec);
  const int64_t len = (int64_t)A->n_rows * A->bs;
  const int restart = o->restart;
  const int k_req = o->k;
  const int m = restart > 0 ? restart : std::max(1, o->max_iters + 1);
  if (restart > 256) {
    record_error("pGMRES restart length above 256 is not supported");
    return BSP_INVALID;
  }
  // Basis vectors.  Restarted: m+1 vectors plus k+2 spares for the deflated
  // restart, allocated once.  Unrestarted: grown in chunks as the space grows.
  constexpr int kChunk = 16;
  const int n_spare = restart > 0 ? std::min(k_req, m) + 2 : 0;
  int n_chunks = 0;
  std::vector<double*> qptr, spare;
  Span<double*> dq, dspare;
  BSP_TRY(h->scratch("gmres.qtab", m + 1, &dq.p));
  BSP_TRY(h->scratch("gmres.sparetab", std::max(n_spare, 1), &dspare.p));
  auto upload_tables = [&]() -> int {
    const int cnt = std::min<int>((int)qptr.size(), m + 1);
    BSP_CUDA_TRY(cudaMemcpyAsync(dq.get(), qptr.data(), cnt * sizeof(double*), cudaMemcpyHostToDevice, h->stream));
    if (n_spare > 0)
      BSP_CUDA_TRY(cudaMemcpyAsync(dspare.get(), spare.data(), n_spare * sizeof(double*), cudaMemcpyHostToDevice, h->stream));
    return BSP_OK;
  };
  auto ensure_basis = [&](int count) -> int {
    bool grew = false;
    while ((int)qptr.size() < count) {
      const int nv = restart > 0 ? (m + 1 + n_spare) : kChunk;
      double* c = nullptr;
      BSP_TRY(h->scratch("gmres.basis." + std::to_string(n_chunks++), (size_t)nv * len, &c));
      for (int t = 0; t < nv; ++t) {
        double* ptr = c + (size_t)t * len;
        if (restart > 0 && t > m) spare.push_back(ptr);
        else qptr.push_back(ptr);
      }
      grew = true;
    }
    if (grew) BSP_TRY(upload_tables());
    return BSP_OK;
  };
  Span<double> vv, vx0, vr0;
  BSP_TRY(h->scratch("gmres.v", len, &vv.p));
  BSP_TRY(h->scratch("gmres.x0", len, &vx0.p));
  BSP_TRY(h->scratch("gmres.r0", len, &vr0.p));
  // small dense state
  const int hcap = std::max(4, o->max_iters + 2 + (restart > 0 ? o->max_iters / restart + 2 : 0));
  const size_t HM = (size_t)(m + 1) * m;
  const size_t nrot_cap = (size_t)(m + 1) * (m + 2) / 2 + m + 8;
  Span<double> dsm;
  size_t dr = restart > 0 ? (size_t)m * m * 3 + (size_t)(m + 1) * (m + 2) + 8 * (size_t)m + 64 + HM : 0;
  const size_t total = 2 * HM + 3 * (size_t)(m + 2) + hcap + dr;
  BSP_TRY(h->scratch("gmres.dense", total, &dsm.p));
  Span<sd::Rot> drots;
  BSP_TRY(h->scratch("gmres.rots", nrot_cap, &drots.p));
  Span<int> dint;
  BSP_TRY(h->scratch("gmres.int", 1 + 2 * (size_t)m + 8, &dint.p));
  Span<KHead> dhead;
  BSP_TRY(h->scratch("gmres.head", 1, &dhead.p));
  Span<double> mgs_part;
  Span<unsigned> mgs_bar;
  BSP_TRY(h->scratch("gmres.mgs_partials", (size_t)(m + 2) * h->num_sms, &mgs_part.p));
  BSP_TRY(h->scratch("gmres.mgs_barrier", 1, &mgs_bar.p));
  BSP_CUDA_TRY(cudaMemsetAsync(dsm.get(), 0, total * sizeof(double), h->stream));
  BSP_CUDA_TRY(cudaMemsetAsync(dhead.get(), 0, sizeof(KHead), h->stream));
  GPtrs gp{};
  gp.head = dhead.get();
  gp.m = m;
  double* base = dsm.get();
  gp.H = base; base += HM;
  gp.R = base; base += HM;
  gp.g = base; base += m + 2;
  gp.rhs = base; base += m + 2;
  gp.y = base; base += m + 2;
  gp.hist = base; base += hcap;
  gp.hist_cap = hcap;
  if (restart > 0) {
    gp.Hn = base; base += (size_t)m * m;
    gp.Z = base; base += (size_t)m * m;
    gp.work = base; base += (size_t)m * m + 4 * (size_t)m + 32;
    gp.P = base; base += (size_t)(m + 1) * (m + 2);
    gp.w = base; base += m + 1;
    gp.wr = base; base += m + 1;
    gp.wi = base; base += m + 1;
    gp.resv = base; base += m + 2;
    gp.Hnew = base; base += HM;
  }
  gp.rots = drots.get();
  gp.nrot = dint.get();
  gp.perm = dint.get() + 1;
  gp.sel = dint.get() + 1 + m;
  KHead* hd = dhead.get();
  const int g = grid_for(h, len, 256);
  size_t defl_smem = 0;
  if (restart > 0 && deflate_smem_bytes(m) <= kDeflateSmemMax) {
    defl_smem = deflate_smem_bytes(m);
    BSP_CUDA_TRY(cudaFuncSetAttribute(k_gm_deflate, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)defl_smem));
  }

  EventTimer tm(h->stream);
  BSP_TRY(ensure_basis(restart > 0 ? m + 1 : 2));
  BSP_CUDA_TRY(cudaMemsetAsync(vx0.get(), 0, len * sizeof(double), h->stream));  // x_0 = 0
  // r_0 = M^-1 b; res_mag[0] = ||r_0||; q_0 = r_0 / res_mag[0]
  if (pc) BSP_TRY(precond_apply(pc, op_prec,b, vr0.get()));
  else bsp::count_launch(), k_copy<<<g, 256, 0, h->stream>>>(len, b, vr0.get());
  BSP_TRY(launch_reduce<1>(h, 7, len, DotBody{vr0.get(), vr0.get()}, NormFin{&hd->res0}));
  bsp::count_launch(), k_div<<<g, 256, 0, h->stream>>>(len, vr0.get(), &hd->res0, hd, qptr[0]);
  bsp::count_launch(), k_gm_init<<<1, 1, 0, h->stream>>>(gp, o->tol);
  BSP_CUDA_TRY(cudaPeekAtLastError());
  KHead st;
  BSP_TRY(read_head(h, hd, &st));
  int n_restarts = 0;
  // first Arnoldi steps reuse the zeroed memset of q_0 normalisation guard
  while (st.done == DONE_RUNNING) {
    const int j = st.j;
    BSP_TRY(ensure_basis(j + 2));
    // v = M^-1 A q_j
    BSP_TRY(bsmv_launch(A, 1, 0, op_dtype, 1.0,qptr[j], 0.0, nullptr, vv.get(), h->stream));
    if (pc) BSP_TRY(precond_apply(pc, op_prec,vv.get(), vv.get()));
    // MGS: one persistent launch when v's slices fit, else j+2 fused passes
    const int mg = launch_mgs(h, len, vv.get(), dq.get(), j, gp.H, m, hd, mgs_part.get(), mgs_bar.get());
    if (mg > 1) return mg;
    if (mg == 1) {
      for (int i = 0; i <= j; ++i) {
        MgsBody body{vv.get(), i > 0 ? qptr[i - 1] : nullptr, qptr[i],
                     i > 0 ? gp.H + (size_t)(i - 1) * m + j : nullptr, 0.0, len};
        BSP_TRY(launch_reduce<1>(h, 8 + (i & 1), chunks_of(len), body, StoreFin{gp.H + (size_t)i * m + j}));
      }
      BSP_TRY(launch_reduce<1>(h, 10, chunks_of(len), MgsLastBody{vv.get(), qptr[j], gp.H + (size_t)j * m + j, 0.0, len},
                               NormFin{gp.H + (size_t)(j + 1) * m + j}));
      bsp::count_launch(), k_div<<<g, 256, 0, h->stream>>>(len, vv.get(), gp.H + (size_t)(j + 1) * m + j, hd, qptr[j + 1]);
    }
    bsp::count_launch(), k_gm_ls<<<1, 1, 0, h->stream>>>(gp, o->max_iters);
    BSP_CUDA_TRY(cudaPeekAtLastError());
    BSP_TRY(read_head(h, hd, &st));
    if (st.done != DONE_RUNNING) break;
    if (restart > 0 && st.j == restart) {
      // x_0 = x_0 + Q y
      bsp::count_launch(), k_gm_y<<<1, 1, 0, h->stream>>>(gp);
      bsp::count_launch(), k_gm_combine<<<g, 256, 0, h->stream>>>(len, vx0.get(), dq.get(), gp.y, hd);
      ++n_restarts;
      if (k_req == 0) {
        // r_0 = M^-1 (b - A x_0), pure restart
        BSP_TRY(bsmv_launch(A, 1, 0, op_dtype, -1.0, vx0.get(), 1.0, b, vr0.get(), h->stream));
        if (pc) BSP_TRY(precond_apply(pc, op_prec,vr0.get(), vr0.get()));
        BSP_TRY(launch_reduce<1>(h, 7, len, DotBody{vr0.get(), vr0.get()}, NormFin{&hd->res0}));
        bsp::count_launch(), k_div<<<g, 256, 0, h->stream>>>(len, vr0.get(), &hd->res0, hd, qptr[0]);
        bsp::count_launch(), k_gm_pure_restart<<<1, 1, 0, h->stream>>>(gp);
      } else {
        bsp::count_launch(), k_gm_deflate<<<1, 32, defl_smem, h->stream>>>(gp, k_req, n_spare, defl_smem > 0);
        bsp::count_launch(), k_gm_qn_update<<<g, 256, (size_t)(st.j + 1) * kQnCols * sizeof(double), h->stream>>>(
            len, dq.get(), dspare.get(), gp.P, m + 1, hd, st.j + 1);
      }
      BSP_CUDA_TRY(cudaPeekAtLastError());
      BSP_TRY(read_head(h, hd, &st));
      if (k_req != 0 && st.done == DONE_RUNNING) {
        if (st.keff + 1 > n_spare) {
          record_error("deflated restart kept more vectors than reserved");
          return BSP_BREAKDOWN;
        }
        for (int c = 0; c <= st.keff; ++c) std::swap(qptr[c], spare[c]);
        BSP_TRY(upload_tables());
      }
    }
  }
  // x = x_0 + Q y
  bsp::count_launch(), k_gm_y<<<1, 1, 0, h->stream>>>(gp);
  BSP_CUDA_TRY(cudaMemcpyAsync(x, vx0.get(), len * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  bsp::count_launch(), k_gm_combine<<<g, 256, 0, h->stream>>>(len, x, dq.get(), gp.y, hd);
  BSP_CUDA_TRY(cudaPeekAtLastError());
  const double solve_ms = tm.stop_ms();
  if (pc) BSP_TRY(precond_check_status(pc));
  const int nh = std::min(st.n_hist, hcap);
  if (hist && hist_cap > 0)
    BSP_CUDA_TRY(cudaMemcpy(hist, gp.hist, std::min(nh, hist_cap) * sizeof(double), cudaMemcpyDeviceToHost));
  if (info) {
    info->status = status_of(st.done);
    info->iters = st.tot;
    info->n_hist = nh;
    info->n_restarts = n_restarts;
    info->res0 = st.res0;
    info->final_res = st.res;
    info->solve_ms = solve_ms;
    if (want_true) BSP_TRY(true_residual(h, A, b, x, vv.get(), &info->true_rel_res));
  }
  if (o->print_iters) {
    printf("pGMRES iters %d\n", st.tot);  // solvers.hpp:266-270
    if (st.tot > o->max_iters) printf("maximum pGMRES iterations reached\n");
  }
  if (o->print_eig_info && st.j > 0) {
    // eigenvalues of the final H's square part; harmonic Ritz values after a
    // restart (solvers.hpp:272-288)
    std::vector<double> wr(st.j), wi(st.j);
    const bool harm = n_restarts > 0;
    BSP_TRY(ritz_values(h, gp.H, m, st.j, harm, wr.data(), wi.data()));
    print_eigs(wr.data(), wi.data(), st.j, harm, true, false);
  }
  return status_of(st.done);
}

int precond_ensure_precision(bsp_precond_s* pc, int precision);

__global__ void k_add(int64_t n, const double* __restrict__ d, double* __restrict__ x) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] += d[i];
}

// FP64 iterative refinement around the Krylov solver.  Used for the true-
// residual stopping rule and for the mixed-precision inner operator:
//   x = 0, r = b;  repeat: solve A d = r (inner tolerance), x += d,
//   r = b - A x in FP64, stop when ||r|| / ||b|| <= tol.
// The inner solve runs the reference's method with the requested operator
// precision; its residual history entries are appended to hist.
int refine_solve(bool gmres, bsp_handle_s* h, bsp_matrix_s* A, bsp_precond_s* pc, const double* b,
                 double* x, const bsp_solve_opts* o, double* hist, int hist_cap, bsp_solve_info* info) {
  const int64_t len = (int64_t)A->n_rows * A->bs;
  const int prec = o->precision;
  if (prec != BSP_PREC_F64) {
    BSP_TRY(bsp_matrix_make_lowp(A, prec == BSP_PREC_F32 ? BSP_F32 : BSP_BF16));
    if (pc) BSP_TRY(precond_ensure_precision(pc, prec));
  }
  Span<double> r, d, work;
  BSP_TRY(h->scratch("refine.r", len, &r.p));
  BSP_TRY(h->scratch("refine.d", len, &d.p));
  BSP_TRY(h->scratch("refine.work", len, &work.p));
  const int g = grid_for(h, len, 256);
  EventTimer tm(h->stream);
  double* sc = h->ws.scalars.get();
  BSP_CUDA_TRY(cudaMemsetAsync(x, 0, len * sizeof(double), h->stream));
  bsp::count_launch(), k_copy<<<g, 256, 0, h->stream>>>(len, b, r.get());
  BSP_TRY(launch_reduce<1>(h, 11, len, DotBody{b, b}, StoreFin{sc + 8}));
  double bb = 0.0;
  BSP_CUDA_TRY(cudaMemcpyAsync(&bb, sc + 8, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  BSP_CUDA_TRY(cudaStreamSynchronize(h->stream));
  const double bnorm = sqrt(bb);
  double rel = 1.0;
  int total_iters = 0, n_hist = 0, n_restarts = 0, outer = 0, status = BSP_MAXIT;
  const int max_outer = o->max_outer > 0 ? o->max_outer : 50;
  if (!(bnorm > 0.0)) {
    status = std::isfinite(bnorm) ? BSP_OK : BSP_NAN;
    rel = 0.0;
  }
  while (status == BSP_MAXIT && outer < max_outer) {
    bsp_solve_opts in = *o;
    in.print_iters = 0;
    if (prec == BSP_PREC_F64)
      in.tol = outer == 0 ? o->tol : std::min(0.5, 0.5 * o->tol / rel);
    else
      in.tol = std::max(o->inner_tol > 0 ? o->inner_tol : 1e-6, 0.5 * o->tol / rel);
    in.max_iters = std::max(1, o->max_iters - total_iters);
    bsp_solve_info ii{};
    const int cap = hist ? std::max(0, hist_cap - n_hist) : 0;
    const int s = gmres ? pgmres_solve(h, A, pc, r.get(), d.get(), &in, hist ? hist + n_hist : nullptr,
                                       cap, &ii, prec, false)
                        : pcg_solve(h, A, pc, r.get(), d.get(), &in, hist ? hist + n_hist : nullptr, cap,
                                    &ii, prec, false);
    total_iters += ii.iters;
    n_hist += std::min(ii.n_hist, cap);
    n_restarts += ii.n_restarts;
    ++outer;
    if (s != BSP_OK && s != BSP_MAXIT && s != BSP_BREAKDOWN) {
      status = s;  // NaN or a device failure: the correction is not usable
      break;
    }
    // x += d.  A Krylov breakdown still leaves the minimiser over the space
    // built so far in d, so it is applied and the true residual recomputed;
    // the solve then stops with BREAKDOWN unless that residual meets tol.
    bsp::count_launch(), k_add<<<g, 256, 0, h->stream>>>(len, d.get(), x);
    // r = b - A x in FP64; rel = ||r|| / ||b||
    BSP_TRY(bsmv_launch(A, 1, 0, BSP_F64, -1.0, x, 1.0, b, r.get(), h->stream));
    BSP_TRY(launch_reduce<1>(h, 12, len, DotBody{r.get(), r.get()}, StoreFin{sc + 9}));
    double rr = 0.0;
    BSP_CUDA_TRY(cudaMemcpyAsync(&rr, sc + 9, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    BSP_CUDA_TRY(cudaStreamSynchronize(h->stream));
    rel = sqrt(rr) / bnorm;
    if (!std::isfinite(rel)) status = BSP_NAN;
    else if (rel <= o->tol) status = BSP_OK;
    else if (s == BSP_BREAKDOWN) status = BSP_BREAKDOWN;
    else if (total_iters >= o->max_iters) break;
  }
  const double ms = tm.stop_ms();
  if (info) {
    info->status = status;
    info->iters = total_iters;
    info->inner_iters = total_iters;
    info->n_outer = outer;
    info->n_hist = n_hist;
    info->n_restarts = n_restarts;
    info->final_res = rel;
    info->true_rel_res = rel;
    info->solve_ms = ms;
  }
  if (o->print_iters) printf("%s iters %d (refinement steps %d)\n", gmres ? "pGMRES" : "pCG", total_iters, outer);
  return status;
}

}  // namespace bsp

// ================================================================== C ABI
using namespace bsp;

namespace bsp {
int pgmres_complex_solve(bsp_handle_s* h, bsp_matrix_s* A, bsp_precond_s* pc, const double* b, double* x,
                         const bsp_solve_opts* o, double* hist, int hist_cap, bsp_solve_info* info);
}  // namespace bsp

static int solve_common(bool gmres, bsp_handle_t h, bsp_matrix_t A, bsp_precond_t pc,
                        const double* b, double* x, const bsp_solve_opts* opts, double* hist,
                        int hist_cap, bsp_solve_info* info) {
  if (!h || !A || !b || !x || !opts) return BSP_INVALID;
  if (A->n_rows != A->n_cols) return BSP_INVALID;
  BSP_CUDA_TRY(cudaSetDevice(h->device));
  if (info) *info = bsp_solve_info{};
  if (A->cbs) {
    // complex T: pGMRES only (no complex pCG in the reference, solvers.hpp:55)
    if (!gmres) {
      record_error("pCG is not defined for complex matrices");
      return BSP_INVALID;
    }
    return pgmres_complex_solve(h, A, pc, b, x, opts, hist, hist_cap, info);
  }
  if (opts->precision != BSP_PREC_F64 || opts->stop_rule == BSP_STOP_TRUE_RESIDUAL)
    return refine_solve(gmres, h, A, pc, b, x, opts, hist, hist_cap, info);
  return gmres ? pgmres_solve(h, A, pc, b, x, opts, hist, hist_cap, info)
               : pcg_solve(h, A, pc, b, x, opts, hist, hist_cap, info);
}

static int solve_host(bool gmres, bsp_handle_t h, bsp_matrix_t A, bsp_precond_t pc,
                      const double* b, double* x, const bsp_solve_opts* opts, double* hist,
                      int hist_cap, bsp_solve_info* info) {
  if (!h || !A || !b || !x) return BSP_INVALID;
  BSP_CUDA_TRY(cudaSetDevice(h->device));
  const size_t len = (size_t)A->n_rows * A->bs;
  BSP_TRY(h->stage(len, len));
  BSP_CUDA_TRY(cudaMemcpyAsync(h->stage_in.get(), b, len * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  const int s = solve_common(gmres, h, A, pc, h->stage_in.get(), h->stage_out.get(), opts, hist,
                             hist_cap, info);
  if (s != BSP_OK && s != BSP_MAXIT && s != BSP_BREAKDOWN && s != BSP_NAN) return s;
  BSP_CUDA_TRY(cudaMemcpyAsync(x, h->stage_out.get(), len * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  BSP_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return s;
}

extern "C" {

int bsp_pcg_dev(bsp_handle_t h, bsp_matrix_t A, bsp_precond_t pc, const double* b, double* x,
                const bsp_solve_opts* opts, double* hist, int hist_cap, bsp_solve_info* info) {
  return solve_common(false, h, A, pc, b, x, opts, hist, hist_cap, info);
}
int bsp_pgmres_dev(bsp_handle_t h, bsp_matrix_t A, bsp_precond_t pc, const double* b, double* x,
                   const bsp_solve_opts* opts, double* hist, int hist_cap, bsp_solve_info* info) {
  return solve_common(true, h, A, pc, b, x, opts, hist, hist_cap, info);
}
int bsp_pcg(bsp_handle_t h, bsp_matrix_t A, bsp_precond_t pc, const double* b, double* x,
            const bsp_solve_opts* opts, double* hist, int hist_cap, bsp_solve_info* info) {
  return solve_host(false, h, A, pc, b, x, opts, hist, hist_cap, info);
}
int bsp_pgmres(bsp_handle_t h, bsp_matrix_t A, bsp_precond_t pc, const double* b, double* x,
               const bsp_solve_opts* opts, double* hist, int hist_cap, bsp_solve_info* info) {
  return solve_host(true, h, A, pc, b, x, opts, hist, hist_cap, info);
}
int bsp_arnoldi_eigenvalues(bsp_handle_t h, bsp_matrix_t A, bsp_precond_t pc, int iters, int harmonic_ritz,
                            int print_info, int print_vals, double* wr, double* wi, int* n_out) {
  if (!h || !A || !wr || !wi || !n_out || iters < 1) return BSP_INVALID;
  if (A->n_rows != A->n_cols) return BSP_INVALID;
  BSP_CUDA_TRY(cudaSetDevice(h->device));
  const int64_t len = (int64_t)A->n_rows * A->bs;
  iters = (int)std::min<int64_t>(iters, len);  // solvers.hpp:323
  const int m = iters;
  double *basis = nullptr, *v = nullptr, *H = nullptr, *part = nullptr;
  double** qtab = nullptr;
  KHead* head = nullptr;
  unsigned* bar = nullptr;
  BSP_TRY(h->scratch("arnoldi.basis", (size_t)(m + 1) * len, &basis));
  BSP_TRY(h->scratch("arnoldi.v", len, &v));
  BSP_TRY(h->scratch("arnoldi.H", (size_t)(m + 1) * m, &H));
  BSP_TRY(h->scratch("arnoldi.qtab", m + 1, &qtab));
  BSP_TRY(h->scratch("arnoldi.head", 1, &head));
  BSP_TRY(h->scratch("arnoldi.partials", (size_t)(m + 2) * h->num_sms, &part));
  BSP_TRY(h->scratch("arnoldi.barrier", 1, &bar));
  std::vector<double*> qp(m + 1);
  for (int i = 0; i <= m; ++i) qp[i] = basis + (size_t)i * len;
  BSP_CUDA_TRY(cudaMemcpyAsync(qtab, qp.data(), (m + 1) * sizeof(double*), cudaMemcpyHostToDevice, h->stream));
  // zero_thresh = 10 M^2 eps (solvers.hpp:320) in the head the MGS kernels read
  KHead hd{};
  hd.zero_thresh = 10.0 * A->bs * A->bs * kEps;
  BSP_CUDA_TRY(cudaMemcpyAsync(head, &hd, sizeof(KHead), cudaMemcpyHostToDevice, h->stream));
  BSP_CUDA_TRY(cudaMemsetAsync(H, 0, (size_t)(m + 1) * m * sizeof(double), h->stream));
  // q_0 = e_0
  BSP_CUDA_TRY(cudaMemsetAsync(qp[0], 0, len * sizeof(double), h->stream));
  const double one = 1.0;
  BSP_CUDA_TRY(cudaMemcpyAsync(qp[0], &one, sizeof(double), cudaMemcpyHostToDevice, h->stream));
  const int g = grid_for(h, len, 256);
  int n = 0;
  for (int it = 0; it < m; ++it) {
    BSP_TRY(bsmv_launch(A, 1, 0, BSP_F64, 1.0, qp[it], 0.0, nullptr, v, h->stream));
    if (pc) BSP_TRY(precond_apply(pc, BSP_PREC_F64, v, v));
    const int mg = launch_mgs(h, len, v, qtab, it, H, m, head, part, bar);
    if (mg > 1) return mg;
    if (mg == 1) {
      for (int i = 0; i <= it; ++i) {
        MgsBody body{v, i > 0 ? qp[i - 1] : nullptr, qp[i], i > 0 ? H + (size_t)(i - 1) * m + it : nullptr, 0.0, len};
        BSP_TRY(launch_reduce<1>(h, 8 + (i & 1), chunks_of(len), body, StoreFin{H + (size_t)i * m + it}));
      }
      BSP_TRY(launch_reduce<1>(h, 10, chunks_of(len), MgsLastBody{v, qp[it], H + (size_t)it * m + it, 0.0, len},
                               NormFin{H + (size_t)(it + 1) * m + it}));
      bsp::count_launch(), k_div<<<g, 256, 0, h->stream>>>(len, v, H + (size_t)(it + 1) * m + it, head, qp[it + 1]);
    }
    n = it + 1;
    double hsub = 0.0;
    BSP_CUDA_TRY(cudaMemcpyAsync(&hsub, H + (size_t)(it + 1) * m + it, sizeof(double), cudaMemcpyDeviceToHost,
                                 h->stream));
    BSP_CUDA_TRY(cudaStreamSynchronize(h->stream));
    if (std::fabs(hsub) < hd.zero_thresh) break;  // the Krylov space is exhausted
  }
  if (pc) BSP_TRY(precond_check_status(pc));
  BSP_TRY(ritz_values(h, H, m, n, harmonic_ritz != 0, wr, wi));
  *n_out = n;
  print_eigs(wr, wi, n, harmonic_ritz != 0, print_info != 0, print_vals != 0);
  return BSP_OK;
}

int bsp_true_residual_dev(bsp_handle_t h, bsp_matrix_t A, const double* b, const double* x,
                          double* rel_res_host) {
  if (!h || !A || !b || !x || !rel_res_host) return BSP_INVALID;
  BSP_CUDA_TRY(cudaSetDevice(h->device));
  double* w = nullptr;
  BSP_TRY(h->scratch("true_residual.w", (size_t)A->n_rows * A->bs, &w));
  return true_residual(h, A, b, x, w, rel_res_host);
}

}  // extern "C"
