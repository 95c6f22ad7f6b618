// complex.cu — the solve path with T = std::complex<double>.
//
// A complex block matrix is held as its real embedding: complex entry
// a = ar + i ai of a bs x bs block becomes the 2 x 2 real block
// [[ar, -ai], [ai, ar]] at rows 2r, 2r+1 and columns 2c, 2c+1 of a 2bs x 2bs
// block, and a complex vector, stored as interleaved (re, im) doubles (the
// std::complex<double> layout), is the real vector the embedded blocks act on.
// The embedding is an algebra homomorphism (sums, products and inverses of
// embedded blocks are embedded blocks), so the real kernels compute, on it,
// exactly the complex operations the reference runs for T = complex<double>:
//   bsmv                        blocksp_multiply.hpp:209-246
//   Diag / SOR / ILU0           blocksp_preconditioners.hpp:75-357 (block
//                               inverses of the embedded blocks = embedded
//                               complex inverses)
// What does not carry over is the Krylov method: real GMRES on the embedded
// system minimises over real coefficients, complex GMRES over complex ones.
// So pGMRES and its deflated restart are restated here in complex arithmetic
// (blocksp_solvers.hpp:107-295, blocksp_deflated_restart.hpp:38-269, complex
// branches): dot(x, y) = sum conj(x_i) y_i (blocksp_utility.hpp:277-292), the
// Arnoldi step on the device (complex dot and axpy kernels over the
// interleaved vectors), the small dense work (least squares, harmonic Ritz
// values, complex Schur form and its reordering) on the host.  The reference
// has no complex pCG / IChol0 (static_asserts at blocksp_solvers.hpp:55, 411,
// 485); neither has this library.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <limits>
#include <vector>
#include "complex_dense.h"
#include "reduce.cuh"
#include "precond.hpp"

namespace bsp {
int bsmv_launch(bsp_matrix_s* A, int nrhs, int transpose, int dtype, double alpha, const void* x, double beta,
                const void* z, void* y, cudaStream_t stream);
int precond_apply(bsp_precond_s* pc, int precision, const void* r, void* z);
int precond_check_status(bsp_precond_s* pc);
int true_residual(bsp_handle_s* h, bsp_matrix_s* A, const double* b, const double* x, double* work,
                  double* rel);
void print_eigs(const double* wr, const double* wi, int n, bool harmonic, bool info, bool vals);
}  // namespace bsp

namespace {

using namespace bsp;
using Cx = std::complex<double>;
using namespace bsp::cd;

// ------------------------------------------------------------------ kernels
// Reduction body: (re, im) of sum conj(x_c) y_c over complex elements c.
struct CDotBody {
  const double2* x;
  const double2* y;
  __device__ void setup() {}
  __device__ void operator()(int64_t c, double (&a)[2]) const {
    const double2 u = x[c], v = y[c];
    a[0] = fma(u.x, v.x, fma(u.y, v.y, a[0]));
    a[1] = fma(u.x, v.y, fma(-u.y, v.x, a[1]));
  }
};
struct Store2Fin {
  double* out;
  __device__ void operator()(const double (&s)[2]) const {
    out[0] = s[0];
    out[1] = s[1];
  }
};
// Reduction body: sum |y_c|^2 = dot(y, y).
struct CNormBody {
  const double2* y;
  __device__ void setup() {}
  __device__ void operator()(int64_t c, double (&a)[1]) const {
    const double2 v = y[c];
    a[0] = fma(v.x, v.x, fma(v.y, v.y, a[0]));
  }
};

// y -= h x with h = (hp[0], hp[1]) read from device memory (the Arnoldi
// coefficient just reduced): axpy(v, -H(j, iter), Qn[j]).
__global__ void k_caxpy_dev(int64_t nc, const double* __restrict__ hp, const double2* __restrict__ x,
                            double2* __restrict__ y) {
  const double hr = -hp[0], hi = -hp[1];
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += (int64_t)gridDim.x * blockDim.x) {
    const double2 u = x[c];
    double2 v = y[c];
    v.x = fma(hr, u.x, fma(-hi, u.y, v.x));
    v.y = fma(hr, u.y, fma(hi, u.x, v.y));
    y[c] = v;
  }
}

// y += a x, a a host scalar (x = x_0 + Q y).
__global__ void k_caxpy(int64_t nc, double ar, double ai, const double2* __restrict__ x, double2* __restrict__ y) {
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += (int64_t)gridDim.x * blockDim.x) {
    const double2 u = x[c];
    double2 v = y[c];
    v.x = fma(ar, u.x, fma(-ai, u.y, v.x));
    v.y = fma(ar, u.y, fma(ai, u.x, v.y));
    y[c] = v;
  }
}

// q = v / d for a real d (block /= H(iter+1, iter) with a real norm).
__global__ void k_cdiv(int64_t n, double d, const double* __restrict__ v, double* __restrict__ q) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    q[i] = v[i] / d;
}

// out_l = sum_i Q_i P(i, l), l < kp1 (Qn_new = Qn P_{k+1}); P row-major m x kp1
// complex; the basis vectors are given by a pointer table.
__global__ void k_cbasis_combine(int64_t nc, int m, int kp1, const double2* const* __restrict__ Q,
                                 const double2* __restrict__ P, double2* const* __restrict__ out) {
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += (int64_t)gridDim.x * blockDim.x)
    for (int l = 0; l < kp1; ++l) {
      double ar = 0.0, ai = 0.0;
      for (int i = 0; i < m; ++i) {
        const double2 q = Q[i][c], p = P[i * kp1 + l];
        ar = fma(q.x, p.x, fma(-q.y, p.y, ar));
        ai = fma(q.x, p.y, fma(q.y, p.x, ai));
      }
      out[l][c] = make_double2(ar, ai);
    }
}

}  // namespace

namespace bsp {

// Complex pGMRES with deflated restart (blocksp_solvers.hpp:156-295 with
// T = std::complex<double>) on the real embedding A of the complex matrix;
// b and x are interleaved complex vectors (A->n_rows * A->bs doubles).
int pgmres_complex_solve(bsp_handle_s* h, bsp_matrix_s* A, bsp_precond_s* pc, const double* b, double* x,
                         const bsp_solve_opts* o, double* hist, int hist_cap, bsp_solve_info* info) {
  const int64_t len = (int64_t)A->n_rows * A->bs;
  const int64_t nc = len / 2;
  const int restart = o->restart, k_req = o->k, max_iters = o->max_iters;
  if (restart > 256) {
    record_error("pGMRES restart length above 256 is not supported");
    return BSP_INVALID;
  }
  if (restart > 0 && k_req < 0) {
    record_error("complex pGMRES with restarts needs k >= 0");
    return BSP_INVALID;
  }
  if (o->precision != BSP_PREC_F64 || o->stop_rule != BSP_STOP_REFERENCE) {
    record_error("complex pGMRES runs in FP64 with the reference's stopping rule");
    return BSP_INVALID;
  }
  const int cols = restart > 0 ? restart + 1 : std::max(1, max_iters + 2);
  std::vector<double*> Q;
  auto basis = [&](int i) -> double* {
    while ((int)Q.size() <= i) {
      double* p = nullptr;
      if (h->scratch("cgmres.q." + std::to_string(Q.size()), len, &p) != BSP_OK) return nullptr;
      Q.push_back(p);
    }
    return Q[i];
  };
  double *w = nullptr, *x0 = nullptr, *r0 = nullptr, *dsc = nullptr, *dP = nullptr;
  double2** dtab = nullptr;
  BSP_TRY(h->scratch("cgmres.w", len, &w));
  BSP_TRY(h->scratch("cgmres.x0", len, &x0));
  BSP_TRY(h->scratch("cgmres.r0", len, &r0));
  BSP_TRY(h->scratch("cgmres.scalars", (size_t)2 * (cols + 2), &dsc));
  std::vector<double> hsc((size_t)2 * (cols + 2));
  const int g = grid_for(h, nc, 256);
  cudaStream_t st = h->stream;
  EventTimer tm(st);
  auto norm_of = [&](const double* v, double* out) -> int {
    BSP_TRY(launch_reduce<1>(h, 0, nc, CNormBody{reinterpret_cast<const double2*>(v)}, StoreFin{dsc}));
    BSP_CUDA_TRY(cudaMemcpyAsync(hsc.data(), dsc, sizeof(double), cudaMemcpyDeviceToHost, st));
    BSP_CUDA_TRY(cudaStreamSynchronize(st));
    *out = std::sqrt(std::fabs(hsc[0]));
    return BSP_OK;
  };
  // r_0 = M^-1 b, q_0 = r_0 / ||r_0||
  BSP_CUDA_TRY(cudaMemcpyAsync(r0, b, len * sizeof(double), cudaMemcpyDeviceToDevice, st));
  if (pc) BSP_TRY(precond_apply(pc, BSP_PREC_F64, r0, r0));
  std::vector<double> res_mag, hv;
  double nr0 = 0.0;
  BSP_TRY(norm_of(r0, &nr0));
  res_mag.push_back(nr0);
  hv.push_back(nr0);
  if (!basis(0)) return BSP_OUT_OF_MEMORY;
  bsp::count_launch(), k_cdiv<<<grid_for(h, len, 256), 256, 0, st>>>(len, res_mag.back(), r0, Q[0]);
  BSP_CUDA_TRY(cudaMemsetAsync(x0, 0, len * sizeof(double), st));
  const double zero_thresh = std::min(res_mag.back() * kEpsC, kEpsC);
  const double tolerance = res_mag.back() * o->tol;
  int iter = 0, tot = 0, n_restarts = 0;
  CMat H(1, 0);
  std::vector<Cx> y, c_r;
  bool restarted = false;
  while (res_mag.back() > tolerance) {
    // one_arnoldi (blocksp_solvers.hpp:109-136)
    const int m = iter + 2, n = iter + 1;
    CMat Hg(m, n);
    for (int i = 0; i < std::min(H.r, m); ++i)
      for (int j = 0; j < std::min(H.c, n); ++j) Hg(i, j) = H(i, j);
    for (int j = 0; j < n - 1; ++j) Hg(m - 1, j) = 0.0;
    H = Hg;
    BSP_TRY(bsmv_launch(A, 1, 0, BSP_F64, 1.0, Q[iter], 0.0, nullptr, w, st));
    if (pc) BSP_TRY(precond_apply(pc, BSP_PREC_F64, w, w));
    for (int j = 0; j <= iter; ++j) {
      BSP_TRY(launch_reduce<2>(h, 0, nc, CDotBody{reinterpret_cast<const double2*>(Q[j]),
                                                  reinterpret_cast<const double2*>(w)},
                               Store2Fin{dsc + 2 * j}));
      bsp::count_launch(), k_caxpy_dev<<<g, 256, 0, st>>>(nc, dsc + 2 * j, reinterpret_cast<const double2*>(Q[j]),
                                                          reinterpret_cast<double2*>(w));
    }
    BSP_TRY(launch_reduce<1>(h, 0, nc, CNormBody{reinterpret_cast<const double2*>(w)},
                             StoreFin{dsc + 2 * (iter + 1)}));
    BSP_CUDA_TRY(cudaMemcpyAsync(hsc.data(), dsc, (size_t)(2 * (iter + 1) + 1) * sizeof(double),
                                 cudaMemcpyDeviceToHost, st));
    BSP_CUDA_TRY(cudaStreamSynchronize(st));
    for (int j = 0; j <= iter; ++j) H(j, iter) = Cx(hsc[2 * j], hsc[2 * j + 1]);
    const double hn = std::sqrt(std::fabs(hsc[2 * (iter + 1)]));
    if (!std::isfinite(hn)) return BSP_NAN;
    H(iter + 1, iter) = hn;
    if (!(hn < zero_thresh)) {
      if (!basis(iter + 1)) return BSP_OUT_OF_MEMORY;
      bsp::count_launch(), k_cdiv<<<grid_for(h, len, 256), 256, 0, st>>>(len, hn, w, Q[iter + 1]);
    }
    // residual: min || c - H y || (c = ||r_0|| e_1, or c_r after a restart)
    std::vector<Cx> rhs(m, Cx(0.0));
    if (!restarted) rhs[0] = res_mag[0];
    else
      for (int i = 0; i < (int)c_r.size() && i < m; ++i) rhs[i] = c_r[i];
    y = lstsq(H, rhs);
    std::vector<Cx> res_vec(rhs);
    for (int i = 0; i < m; ++i)
      for (int j = 0; j < n; ++j) res_vec[i] -= H(i, j) * y[j];
    double r = 0.0;
    for (const Cx& v : res_vec) r += std::abs(std::conj(v) * v);
    res_mag.push_back(std::sqrt(r));
    hv.push_back(res_mag.back());
    ++iter;
    ++tot;
    if (tot > max_iters) break;
    if (iter == restart && res_mag.back() > tolerance) {
      // x_0 = x_0 + Q y; r_0 = M^-1 (b - A x_0)
      for (int i = 0; i < (int)y.size(); ++i)
        bsp::count_launch(), k_caxpy<<<g, 256, 0, st>>>(nc, y[i].real(), y[i].imag(),
                                                        reinterpret_cast<const double2*>(Q[i]),
                                                        reinterpret_cast<double2*>(x0));
      BSP_TRY(bsmv_launch(A, 1, 0, BSP_F64, -1.0, x0, 1.0, b, r0, st));
      if (pc) BSP_TRY(precond_apply(pc, BSP_PREC_F64, r0, r0));
      ++n_restarts;
      const int k = std::min(k_req, H.c);
      if (k == 0) {  // pure restart
        H = CMat(1, 0);
        res_mag.clear();
        double nr = 0.0;
        BSP_TRY(norm_of(r0, &nr));
        res_mag.push_back(nr);  // not a printed residual (blocksp_solvers.hpp:256-262)
        c_r.assign(1, Cx(nr));
        bsp::count_launch(), k_cdiv<<<grid_for(h, len, 256), 256, 0, st>>>(len, nr, r0, Q[0]);
        iter = 0;
        restarted = false;
      } else {
        if ((int)Q.size() < H.r) return BSP_BREAKDOWN;  // the last Arnoldi step broke down
        CMat Pk1, Hnew;
        if (deflate_complex(H, res_vec, k, Pk1, Hnew, c_r) != 0) {
          record_error("deflated restart: the complex Schur iteration did not converge");
          return BSP_BREAKDOWN;
        }
        const int kk = Hnew.c, mrows = H.r;
        // Qn_new = Qn P_{k+1}, written to spare vectors, then swapped in
        std::vector<double*> spare(kk + 1);
        for (int l = 0; l <= kk; ++l)
          BSP_TRY(h->scratch("cgmres.spare." + std::to_string(l), len, &spare[l]));
        BSP_TRY(h->scratch("cgmres.P", (size_t)2 * mrows * (kk + 1), &dP));
        BSP_TRY(h->scratch("cgmres.tab", (size_t)(mrows + kk + 1), &dtab));
        std::vector<double2*> tab(mrows + kk + 1);
        for (int i = 0; i < mrows; ++i) tab[i] = reinterpret_cast<double2*>(Q[i]);
        for (int l = 0; l <= kk; ++l) tab[mrows + l] = reinterpret_cast<double2*>(spare[l]);
        BSP_CUDA_TRY(cudaMemcpyAsync(dtab, tab.data(), tab.size() * sizeof(double2*), cudaMemcpyHostToDevice, st));
        BSP_CUDA_TRY(cudaMemcpyAsync(dP, Pk1.a.data(), (size_t)2 * mrows * (kk + 1) * sizeof(double),
                                     cudaMemcpyHostToDevice, st));
        bsp::count_launch(), k_cbasis_combine<<<g, 256, 0, st>>>(nc, mrows, kk + 1, dtab,
                                                                 reinterpret_cast<const double2*>(dP), dtab + mrows);
        BSP_CUDA_TRY(cudaPeekAtLastError());
        for (int l = 0; l <= kk; ++l)
          BSP_CUDA_TRY(cudaMemcpyAsync(Q[l], spare[l], len * sizeof(double), cudaMemcpyDeviceToDevice, st));
        H = Hnew;
        res_mag.assign(1, res_mag.back());
        iter = kk;
        restarted = true;
      }
    }
  }
  // x = x_0 + Q y
  BSP_CUDA_TRY(cudaMemcpyAsync(x, x0, len * sizeof(double), cudaMemcpyDeviceToDevice, st));
  for (int i = 0; i < (int)y.size(); ++i)
    bsp::count_launch(), k_caxpy<<<g, 256, 0, st>>>(nc, y[i].real(), y[i].imag(),
                                                    reinterpret_cast<const double2*>(Q[i]),
                                                    reinterpret_cast<double2*>(x));
  BSP_CUDA_TRY(cudaPeekAtLastError());
  const double solve_ms = tm.stop_ms();
  if (pc) BSP_TRY(precond_check_status(pc));
  const int status = tot > max_iters ? BSP_MAXIT : BSP_OK;
  const int nh = (int)hv.size();
  if (hist && hist_cap > 0) std::copy(hv.begin(), hv.begin() + std::min(nh, hist_cap), hist);
  if (info) {
    info->status = status;
    info->iters = tot;
    info->n_hist = nh;
    info->n_restarts = n_restarts;
    info->res0 = hv[0];
    info->final_res = hv.back();
    info->solve_ms = solve_ms;
    BSP_TRY(true_residual(h, A, b, x, w, &info->true_rel_res));
  }
  if (o->print_iters) {
    printf("pGMRES iters %d\n", tot);
    if (tot > max_iters) printf("maximum pGMRES iterations reached\n");
  }
  if (o->print_eig_info && H.c > 0 && H.r == H.c + 1) {
    // eigenvalues of the final H's square part, harmonic Ritz values after a
    // deflated restart (blocksp_solvers.hpp:272-288; Eigenvalues_Arr, complex
    // branch, blocksp_dense_solvers.hpp:919-965)
    std::vector<Cx> ev;
    if (ritz_values(H, restarted, ev)) {
      const int n = (int)ev.size();
      std::vector<double> wr(n), wi(n);
      for (int i = 0; i < n; ++i) {
        wr[i] = ev[i].real();
        wi[i] = ev[i].imag();
      }
      print_eigs(wr.data(), wi.data(), n, restarted, true, false);
    }
  }
  return status;
}

}  // namespace bsp

// ================================================================= C ABI
extern "C" {

int bsp_matrix_create_complex(bsp_handle_t h, int n_rows, int n_cols, int bs, int64_t nnzb, const int* row_ptr,
                              const int* col_idx, const double* vals, bsp_matrix_t* out) {
  if (!h || !out || bs < 1 || bs > 16 || nnzb < 0 || (nnzb > 0 && !vals)) return BSP_INVALID;
  *out = nullptr;
  const int rb = 2 * bs;
  std::vector<double> emb((size_t)nnzb * rb * rb);
  for (int64_t t = 0; t < nnzb; ++t) {
    const double* src = vals + (size_t)t * bs * bs * 2;
    double* dst = emb.data() + (size_t)t * rb * rb;
    for (int r = 0; r < bs; ++r)
      for (int c = 0; c < bs; ++c) {
        const double ar = src[2 * (r * bs + c)], ai = src[2 * (r * bs + c) + 1];
        dst[(2 * r) * rb + 2 * c] = ar;
        dst[(2 * r) * rb + 2 * c + 1] = -ai;
        dst[(2 * r + 1) * rb + 2 * c] = ai;
        dst[(2 * r + 1) * rb + 2 * c + 1] = ar;
      }
  }
  BSP_TRY(bsp_matrix_create(h, n_rows, n_cols, rb, nnzb, row_ptr, col_idx, emb.data(), out));
  (*out)->cbs = bs;
  return BSP_OK;
}

int bsp_matrix_complex_bs(bsp_matrix_t A, int* complex_bs) {
  if (!A || !complex_bs) return BSP_INVALID;
  *complex_bs = A->cbs;
  return BSP_OK;
}

}  // extern "C"
