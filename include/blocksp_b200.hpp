// blocksp_b200.hpp — C++ drop-in for BlockSp's solve path on the B200 library.
//
// Include the reference's own containers first (blocksp_include.hpp, which
// defines BlockSp::BlockSp<T,N> and BlockSp::solArray<T,B,D>), then this
// header, and swap the namespace of the solve calls:
//
//     BlockSp::ILU0_pGMRES<double,4,2> s(A, 1e-10, 5000, 30, 10);    // CPU
//     blocksp_b200::ILU0_pGMRES<double,4,2> s(A, 1e-10, 5000, 30, 10);  // GPU
//     x = s.solve(A, b);
//
// Names, template parameters, constructor defaults and solve() signatures are
// those of blocksp_solvers.hpp:344-649 (solver structs and ez::), :51-105
// (pCG), :156-295 (pGMRES), blocksp_preconditioners.hpp:75-538
// (preconditioners) and blocksp_multiply.hpp:364-404 (bsmv).  T is double, or
// std::complex<double> for bsmv, Diag / SOR / ILU0 and pGMRES (the reference's
// complex set: no complex pCG or IChol0, blocksp_solvers.hpp:55, 411, 485).
// The matrix is uploaded once, when a preconditioner or solver struct is
// constructed (the reference's structs build their preconditioner in the
// constructor too); solve() uploads b and returns x by value.  Errors that the
// reference would ignore or std::exit on are thrown as blocksp_b200::error.
//
// Only the C ABI (blocksp_b200.h) is used underneath; link with
// -lblocksp_b200.
#pragma once
#include <algorithm>
#include <cmath>
#include <complex>
#include <memory>
#include <type_traits>
#include <stdexcept>
#include <string>
#include <vector>

#include "blocksp_b200.h"

namespace blocksp_b200 {

// ScalarType_t of the reference (blocksp_utility.hpp): the real type under T.
template <typename T> struct scalar_of { using type = T; };
template <typename U> struct scalar_of<std::complex<U>> { using type = U; };
template <typename T> using Scalar = typename scalar_of<T>::type;
template <typename T> constexpr bool is_cplx = !std::is_same_v<T, Scalar<T>>;
// doubles per element of T in the library's vectors (complex: re, im)
template <typename T> constexpr int kWords = is_cplx<T> ? 2 : 1;

struct error : std::runtime_error {
  int status;
  error(int st, const std::string& what) : std::runtime_error(what), status(st) {}
};

inline void check(int st, const char* what, bsp_handle_t h = nullptr) {
  if (st == BSP_OK) return;
  throw error(st, std::string(what) + ": " + bsp_status_string(st) + " (" + bsp_last_error(h) + ")");
}

// One CUDA device + stream; shared by every object built on it.
class Handle {
 public:
  explicit Handle(int device = 0, void* stream = nullptr) {
    check(bsp_handle_create(device, stream, &h_), "bsp_handle_create");
  }
  ~Handle() { bsp_handle_destroy(h_); }
  Handle(const Handle&) = delete;
  Handle& operator=(const Handle&) = delete;
  bsp_handle_t get() const { return h_; }
  static std::shared_ptr<Handle> shared() {
    static std::shared_ptr<Handle> def = std::make_shared<Handle>(0);
    return def;
  }

 private:
  bsp_handle_t h_ = nullptr;
};

// BlockSp<T,N> packed into device BSR (blocksp_containers.hpp:92-496:
// rows of TinyMatrix blocks, get_data(i) / get_colIndex(i)).
class DeviceMatrix {
 public:
  template <class BlockSpT>
  DeviceMatrix(const BlockSpT& A, int N, std::shared_ptr<Handle> h = Handle::shared()) : h_(std::move(h)) {
    using V = std::remove_cv_t<std::remove_pointer_t<decltype(A.get_data(0)[0].data())>>;
    constexpr int W = kWords<V>;
    std::vector<int> row_ptr{0}, col_idx;
    std::vector<double> vals;
    for (int i = 0; i < A.m(); ++i) {
      const auto& blocks = A.get_data(i);
      const auto& cols = A.get_colIndex(i);
      for (size_t t = 0; t < blocks.size(); ++t) {
        col_idx.push_back(cols[t]);
        // row-major TinyMatrix<T,N,N>; complex as interleaved (re, im)
        const double* p = reinterpret_cast<const double*>(blocks[t].data());
        vals.insert(vals.end(), p, p + W * N * N);
      }
      row_ptr.push_back((int)col_idx.size());
    }
    if constexpr (W == 2)
      check(bsp_matrix_create_complex(h_->get(), A.m(), A.n(), N, (int64_t)col_idx.size(), row_ptr.data(),
                                      col_idx.data(), vals.data(), &m_),
            "bsp_matrix_create_complex", h_->get());
    else
      check(bsp_matrix_create(h_->get(), A.m(), A.n(), N, (int64_t)col_idx.size(), row_ptr.data(),
                              col_idx.data(), vals.data(), &m_),
            "bsp_matrix_create", h_->get());
  }
  ~DeviceMatrix() { bsp_matrix_destroy(m_); }
  DeviceMatrix(const DeviceMatrix&) = delete;
  DeviceMatrix& operator=(const DeviceMatrix&) = delete;
  bsp_matrix_t get() const { return m_; }
  bsp_handle_t handle() const { return h_->get(); }

 private:
  std::shared_ptr<Handle> h_;
  bsp_matrix_t m_ = nullptr;
};

// solArray<T,B,D> <-> its (element, dim, b) values (blocksp_containers.hpp:572-736;
// element access x(i, d)(b), since the container's data() is not usable
// through a non-const reference).
template <typename T, int B, int D> std::vector<double> flat(const BlockSp::solArray<T, B, D>& x) {
  std::vector<double> v((size_t)x.len() * B * D * kWords<T>);
  for (int i = 0; i < x.len(); ++i)
    for (int d = 0; d < D; ++d)
      for (int b = 0; b < B; ++b) {
        const size_t e = ((size_t)i * D + d) * B + b;
        if constexpr (is_cplx<T>) {
          v[2 * e] = std::real(x(i, d)(b));
          v[2 * e + 1] = std::imag(x(i, d)(b));
        } else {
          v[e] = x(i, d)(b);
        }
      }
  return v;
}
template <typename T, int B, int D> BlockSp::solArray<T, B, D> unflat(const std::vector<double>& v, int n) {
  BlockSp::solArray<T, B, D> x(n);
  for (int i = 0; i < n; ++i)
    for (int d = 0; d < D; ++d)
      for (int b = 0; b < B; ++b) {
        const size_t e = ((size_t)i * D + d) * B + b;
        if constexpr (is_cplx<T>) x(i, d)(b) = T(v[2 * e], v[2 * e + 1]);
        else x(i, d)(b) = v[e];
      }
  return x;
}

// ---------------------------------------------------------------- bsmv
// b = A x (blocksp_multiply.hpp:364-404): the BlockSp<T,B*D> x solArray<T,B,D>
// (coupled) form.
template <typename T, int B, int D>
BlockSp::solArray<T, B, D> bsmv(const BlockSp::BlockSp<T, B * D>& A, const BlockSp::solArray<T, B, D>& x) {
  DeviceMatrix M(A, B * D);
  const std::vector<double> xv = flat(x);
  std::vector<double> yv((size_t)A.m() * B * D * kWords<T>);
  check(bsp_bsmv(M.handle(), M.get(), 1, 0, 1.0, xv.data(), 0.0, yv.data()), "bsp_bsmv", M.handle());
  return unflat<T, B, D>(yv, A.m());
}

// ---------------------------------------------------------------- preconditioners
// A device preconditioner built from A (the reference keeps a pointer to A,
// preconditioners.hpp:80, 120; here the matrix is uploaded and owned).
template <typename T, int B, int D>
class DevicePrecond {
 public:
  DevicePrecond(const BlockSp::BlockSp<T, B * D>& A, int kind, double w = 1.6, int nu = 3, int type = 0)
      : M_(std::make_shared<DeviceMatrix>(A, B * D)) {
    bsp_precond_params p{kind, w, nu, type, BSP_PREC_F64};
    check(bsp_precond_create(M_->handle(), M_->get(), &p, &pc_), "bsp_precond_create", M_->handle());
  }
  ~DevicePrecond() { bsp_precond_destroy(pc_); }
  DevicePrecond(const DevicePrecond&) = delete;
  DevicePrecond& operator=(const DevicePrecond&) = delete;
  // operator()(solArray&): x <- M^-1 x (preconditioners.hpp:541-556)
  void operator()(BlockSp::solArray<T, B, D>& x) const {
    std::vector<double> v = flat(x);
    check(bsp_precond_apply(M_->handle(), pc_, v.data()), "bsp_precond_apply", M_->handle());
    x = unflat<T, B, D>(v, x.len());
  }
  bsp_precond_t get() const { return pc_; }
  const std::shared_ptr<DeviceMatrix>& matrix() const { return M_; }

 private:
  std::shared_ptr<DeviceMatrix> M_;
  bsp_precond_t pc_ = nullptr;
};

namespace preConditioners {
template <typename T, int B, int D = 1> struct ILU0 : DevicePrecond<T, B, D> {
  explicit ILU0(const BlockSp::BlockSp<T, B * D>& A) : DevicePrecond<T, B, D>(A, BSP_PC_ILU0) {}
};
template <typename T, int B, int D = 1> struct IChol0 : DevicePrecond<T, B, D> {
  explicit IChol0(const BlockSp::BlockSp<T, B * D>& A) : DevicePrecond<T, B, D>(A, BSP_PC_ICHOL0) {}
};
// Diag<Inv,...> with Inv = LU (getrs) or Cholesky (pptrs) block inversion
template <typename T, int B, int D = 1> struct DiagLU : DevicePrecond<T, B, D> {
  explicit DiagLU(const BlockSp::BlockSp<T, B * D>& A) : DevicePrecond<T, B, D>(A, BSP_PC_DIAG_LU) {}
};
template <typename T, int B, int D = 1> struct DiagChol : DevicePrecond<T, B, D> {
  explicit DiagChol(const BlockSp::BlockSp<T, B * D>& A) : DevicePrecond<T, B, D>(A, BSP_PC_DIAG_CHOL) {}
};
template <typename T, int B, int D = 1> struct SORLU : DevicePrecond<T, B, D> {
  SORLU(const BlockSp::BlockSp<T, B * D>& A, double w, int nu, int SORtype = 0)
      : DevicePrecond<T, B, D>(A, BSP_PC_SOR_LU, w, nu, SORtype) {}
};
template <typename T, int B, int D = 1> struct SORChol : DevicePrecond<T, B, D> {
  SORChol(const BlockSp::BlockSp<T, B * D>& A, double w, int nu, int SORtype = 0)
      : DevicePrecond<T, B, D>(A, BSP_PC_SOR_CHOL, w, nu, SORtype) {}
};
}  // namespace preConditioners

// ---------------------------------------------------------------- Krylov
// pCG<T,B,D>(A, b, tol, preCond, maxIters, printIters) (solvers.hpp:51-105);
// the preconditioner carries the device copy of A.
template <typename T, int B, int D>
BlockSp::solArray<T, B, D> pCG(const BlockSp::BlockSp<T, B * D>& A, const BlockSp::solArray<T, B, D>& b, Scalar<T> tol,
                               const DevicePrecond<T, B, D>& preCond, int maxIters = 1000, bool printIters = false,
                               bsp_solve_info* info = nullptr) {
  (void)A;
  static_assert(!is_cplx<T>, "pCG is defined for real T only (blocksp_solvers.hpp:55)");
  const std::vector<double> bv = flat(b);
  std::vector<double> xv(bv.size());
  bsp_solve_opts o{tol, maxIters, -1, -1, printIters ? 1 : 0, BSP_STOP_REFERENCE, BSP_PREC_F64, 1e-6, 50};
  bsp_solve_info local{};
  const int st = bsp_pcg(preCond.matrix()->handle(), preCond.matrix()->get(), preCond.get(), bv.data(), xv.data(),
                         &o, nullptr, 0, info ? info : &local);
  if (st != BSP_OK && st != BSP_MAXIT) check(st, "bsp_pcg", preCond.matrix()->handle());
  return unflat<T, B, D>(xv, b.len());
}

// pGMRES<T,B,D>(A, b, tol, preCond, maxIters, restart, k, printIters,
// printEigInfo) (solvers.hpp:156-295).
template <typename T, int B, int D>
BlockSp::solArray<T, B, D> pGMRES(const BlockSp::BlockSp<T, B * D>& A, const BlockSp::solArray<T, B, D>& b, Scalar<T> tol,
                                  const DevicePrecond<T, B, D>& preCond, int maxIters = 500, int restart = -1,
                                  int k = -1, bool printIters = false, bool printEigInfo = false,
                                  bsp_solve_info* info = nullptr) {
  (void)A;
  const std::vector<double> bv = flat(b);
  std::vector<double> xv(bv.size());
  bsp_solve_opts o{tol,  maxIters, restart, k, printIters ? 1 : 0, BSP_STOP_REFERENCE, BSP_PREC_F64, 1e-6, 50,
                   printEigInfo ? 1 : 0};
  bsp_solve_info local{};
  const int st = bsp_pgmres(preCond.matrix()->handle(), preCond.matrix()->get(), preCond.get(), bv.data(),
                            xv.data(), &o, nullptr, 0, info ? info : &local);
  if (st != BSP_OK && st != BSP_MAXIT && st != BSP_BREAKDOWN) check(st, "bsp_pgmres", preCond.matrix()->handle());
  return unflat<T, B, D>(xv, b.len());
}

// ---------------------------------------------------------------- solver structs
template <typename T, int B, int D = 1>
struct ILU0_pGMRES {
  preConditioners::ILU0<T, B, D> ILU0_pre;
  Scalar<T> tol;
  int maxIters, restart, k;
  bool printIters, printEigInfo;
  ILU0_pGMRES(const BlockSp::BlockSp<T, B * D>& A, Scalar<T> tol = 1.0e-8, int maxIters = 5000, int restart = -1, int k = -1,
              bool printIters = false, bool printEigInfo = false)
      : ILU0_pre(A), tol(tol), maxIters(maxIters), restart(restart), k(k), printIters(printIters),
        printEigInfo(printEigInfo) {}
  BlockSp::solArray<T, B, D> solve(const BlockSp::BlockSp<T, B * D>& A, const BlockSp::solArray<T, B, D>& b) const {
    return pGMRES<T, B, D>(A, b, tol, ILU0_pre, maxIters, restart, k, printIters, printEigInfo);
  }
};

template <typename T, int B, int D = 1>
struct IChol0_pCG {
  preConditioners::IChol0<T, B, D> IChol0_pre;
  Scalar<T> tol;
  int maxIters;
  bool printIters;
  IChol0_pCG(const BlockSp::BlockSp<T, B * D>& A, Scalar<T> tol = 1.0e-8, int maxIters = 5000, bool printIters = false)
      : IChol0_pre(A), tol(tol), maxIters(maxIters), printIters(printIters) {}
  BlockSp::solArray<T, B, D> solve(const BlockSp::BlockSp<T, B * D>& A, const BlockSp::solArray<T, B, D>& b) const {
    return pCG<T, B, D>(A, b, tol, IChol0_pre, maxIters, printIters);
  }
};

template <typename T, int B, int D = 1>
struct SOR_pGMRES {
  preConditioners::SORLU<T, B, D> SOR_pre;
  Scalar<T> tol;
  int maxIters, restart, k;
  bool printIters, printEigInfo;
  SOR_pGMRES(const BlockSp::BlockSp<T, B * D>& A, Scalar<T> w = 1.6, int nu = 3, int SORtype = 0, Scalar<T> tol = 1.0e-8,
             int maxIters = 5000, int restart = -1, int k = -1, bool printIters = false, bool printEigInfo = false)
      : SOR_pre(A, w, nu, SORtype), tol(tol), maxIters(maxIters), restart(restart), k(k), printIters(printIters),
        printEigInfo(printEigInfo) {}
  BlockSp::solArray<T, B, D> solve(const BlockSp::BlockSp<T, B * D>& A, const BlockSp::solArray<T, B, D>& b) const {
    return pGMRES<T, B, D>(A, b, tol, SOR_pre, maxIters, restart, k, printIters, printEigInfo);
  }
};

template <typename T, int B, int D = 1>
struct SOR_pCG {
  preConditioners::SORChol<T, B, D> SOR_pre;
  Scalar<T> tol;
  int maxIters;
  bool printIters;
  SOR_pCG(const BlockSp::BlockSp<T, B * D>& A, Scalar<T> w = 1.6, int nu = 3, Scalar<T> tol = 1.0e-8, int maxIters = 5000,
          bool printIters = false)
      : SOR_pre(A, w, nu, 0), tol(tol), maxIters(maxIters), printIters(printIters) {}
  BlockSp::solArray<T, B, D> solve(const BlockSp::BlockSp<T, B * D>& A, const BlockSp::solArray<T, B, D>& b) const {
    return pCG<T, B, D>(A, b, tol, SOR_pre, maxIters, printIters);
  }
};

// ez:: one-call forms with the reference's packaged defaults (solvers.hpp:508-649)
namespace ez {
template <typename T, int B, int D = 1>
BlockSp::solArray<T, B, D> sor_pGMRES(const BlockSp::BlockSp<T, B * D>& A, const BlockSp::solArray<T, B, D>& b,
                                      bool printIters = false) {
  return SOR_pGMRES<T, B, D>(A, 1.6, 3, 0, 1.0e-8, 5000, -1, -1, printIters).solve(A, b);
}
template <typename T, int B, int D = 1>
BlockSp::solArray<T, B, D> sor_pGMRES_robust(const BlockSp::BlockSp<T, B * D>& A,
                                             const BlockSp::solArray<T, B, D>& b, bool printIters = false) {
  return SOR_pGMRES<T, B, D>(A, 0.6, 3, 0, 1.0e-8, 5000, -1, -1, printIters).solve(A, b);
}
template <typename T, int B, int D = 1>
BlockSp::solArray<T, B, D> sor_pGMRES_dr(const BlockSp::BlockSp<T, B * D>& A, const BlockSp::solArray<T, B, D>& b,
                                         bool printIters = false) {
  return SOR_pGMRES<T, B, D>(A, 1.6, 3, 0, 1.0e-8, 5000, 30, 10, printIters).solve(A, b);
}
template <typename T, int B, int D = 1>
BlockSp::solArray<T, B, D> ilu0_pGMRES(const BlockSp::BlockSp<T, B * D>& A, const BlockSp::solArray<T, B, D>& b,
                                       bool printIters = false) {
  return ILU0_pGMRES<T, B, D>(A, 1.0e-8, 5000, -1, -1, printIters).solve(A, b);
}
template <typename T, int B, int D = 1>
BlockSp::solArray<T, B, D> ilu0_pGMRES_dr(const BlockSp::BlockSp<T, B * D>& A, const BlockSp::solArray<T, B, D>& b,
                                          bool printIters = false) {
  return ILU0_pGMRES<T, B, D>(A, 1.0e-8, 5000, 30, 10, printIters).solve(A, b);
}
template <typename T, int B, int D = 1>
BlockSp::solArray<T, B, D> sor_pCG(const BlockSp::BlockSp<T, B * D>& A, const BlockSp::solArray<T, B, D>& b,
                                   bool printIters = false) {
  return SOR_pCG<T, B, D>(A, 1.6, 3, 1.0e-8, 5000, printIters).solve(A, b);
}
template <typename T, int B, int D = 1>
BlockSp::solArray<T, B, D> ichol0_pCG(const BlockSp::BlockSp<T, B * D>& A, const BlockSp::solArray<T, B, D>& b,
                                      bool printIters = false) {
  return IChol0_pCG<T, B, D>(A, 1.0e-8, 5000, printIters).solve(A, b);
}
}  // namespace ez

// ---------------------------------------------------------------- block algebra
// bs_id, bs_tr, bsmm (blocksp_multiply.hpp:335-362) on the reference's
// container: computed on the GPU, returned as a host BlockSp<T,M> whose rows
// list their blocks in the order the reference's loops create them.
namespace detail {
// Owns a device matrix made by the library.
struct OwnedMatrix {
  bsp_matrix_t m = nullptr;
  ~OwnedMatrix() { bsp_matrix_destroy(m); }
};
template <typename T, int M> BlockSp::BlockSp<T, M> to_blocksp(bsp_matrix_t C) {
  int n = 0, nc = 0, bs = 0;
  int64_t nnzb = 0;
  check(bsp_matrix_info(C, &n, &nc, &bs, &nnzb), "bsp_matrix_info");
  std::vector<int> rp(n + 1), ci(nnzb > 0 ? nnzb : 1);
  std::vector<double> v((size_t)(nnzb > 0 ? nnzb : 1) * M * M);
  check(bsp_matrix_export(C, rp.data(), ci.data(), v.data()), "bsp_matrix_export");
  BlockSp::BlockSp<T, M> out(n, nc);
  for (int i = 0; i < n; ++i)
    for (int t = rp[i]; t < rp[i + 1]; ++t) {
      blitz::TinyMatrix<T, M, M> blk;
      for (int e = 0; e < M * M; ++e) blk.data()[e] = v[(size_t)t * M * M + e];
      out(i, ci[t]) = blk;
    }
  return out;
}
}  // namespace detail

template <typename T, int M> BlockSp::BlockSp<T, M> bs_id(int size) {
  auto h = Handle::shared();
  detail::OwnedMatrix C;
  check(bsp_bs_id(h->get(), size, M, &C.m), "bsp_bs_id", h->get());
  return detail::to_blocksp<T, M>(C.m);
}

template <typename T, int M> BlockSp::BlockSp<T, M> bs_tr(const BlockSp::BlockSp<T, M>& A) {
  DeviceMatrix dA(A, M);
  detail::OwnedMatrix C;
  check(bsp_bs_tr(dA.handle(), dA.get(), &C.m), "bsp_bs_tr", dA.handle());
  return detail::to_blocksp<T, M>(C.m);
}

template <typename T, int M>
BlockSp::BlockSp<T, M> bsmm(const BlockSp::BlockSp<T, M>& A, const BlockSp::BlockSp<T, M>& B, bool Atran = false) {
  DeviceMatrix dA(A, M), dB(B, M);
  detail::OwnedMatrix C;
  check(bsp_bsmm(dA.handle(), dA.get(), dB.get(), Atran ? 1 : 0, &C.m), "bsp_bsmm", dA.handle());
  return detail::to_blocksp<T, M>(C.m);
}
// triple and quadruple products nest to the right (blocksp_multiply.hpp:137-159)
template <typename T, int M>
BlockSp::BlockSp<T, M> bsmm(const BlockSp::BlockSp<T, M>& A, const BlockSp::BlockSp<T, M>& B,
                            const BlockSp::BlockSp<T, M>& C, bool Atran = false) {
  return bsmm<T, M>(A, bsmm<T, M>(B, C), Atran);
}
template <typename T, int M>
BlockSp::BlockSp<T, M> bsmm(const BlockSp::BlockSp<T, M>& A, const BlockSp::BlockSp<T, M>& B,
                            const BlockSp::BlockSp<T, M>& C, const BlockSp::BlockSp<T, M>& D, bool Atran = false) {
  return bsmm<T, M>(A, bsmm<T, M>(B, C, D), Atran);
}

// ---------------------------------------------------------------- MatrixMarket files
// mtxMatrix_to_BlockSp / mtxArray_to_solArray (blocksp_tests.hpp:582-699)
// through the library's readers (D > 1 vectors are placed correctly).
template <typename T, int B>
BlockSp::BlockSp<T, B> mtxMatrix_to_BlockSp(const std::string& path, unsigned start_line = 0, bool symmetric = false,
                                            bool base_zero = false) {
  int n = 0, nc = 0;
  int64_t nnzb = 0;
  check(bsp_mtx_read_matrix(path.c_str(), B, (int)start_line, symmetric, base_zero, &n, &nc, &nnzb, nullptr,
                            nullptr, nullptr),
        "bsp_mtx_read_matrix");
  std::vector<int> rp(n + 1), ci(nnzb > 0 ? nnzb : 1);
  std::vector<double> v((size_t)(nnzb > 0 ? nnzb : 1) * B * B);
  check(bsp_mtx_read_matrix(path.c_str(), B, (int)start_line, symmetric, base_zero, &n, &nc, &nnzb, rp.data(),
                            ci.data(), v.data()),
        "bsp_mtx_read_matrix");
  BlockSp::BlockSp<T, B> A(n, nc);
  for (int i = 0; i < n; ++i)
    for (int t = rp[i]; t < rp[i + 1]; ++t) {
      blitz::TinyMatrix<T, B, B> blk;
      for (int e = 0; e < B * B; ++e) blk.data()[e] = v[(size_t)t * B * B + e];
      A(i, ci[t]) = blk;
    }
  return A;
}
template <typename T, int B, int D = 1>
BlockSp::solArray<T, B, D> mtxArray_to_solArray(const std::string& path, unsigned start_line = 0) {
  int64_t m = 0;
  check(bsp_mtx_read_vector(path.c_str(), (int)start_line, B, D, &m, nullptr), "bsp_mtx_read_vector");
  std::vector<double> v(m);
  check(bsp_mtx_read_vector(path.c_str(), (int)start_line, B, D, &m, v.data()), "bsp_mtx_read_vector");
  return unflat<T, B, D>(v, (int)(m / (B * D)));
}

// ---------------------------------------------------------------- eigenvalues
// Eigenvalues_Arr (blocksp_dense_solvers.hpp:909-1000) of arnoldi_eigenvalues
// (blocksp_solvers.hpp:306-334), computed on the GPU.
struct Eigenvalues {
  std::vector<double> WR, WI, WM;
  bool harmonic_Ritz = false;
  double min_real() const { return *std::min_element(WR.begin(), WR.end()); }
  double max_real() const { return *std::max_element(WR.begin(), WR.end()); }
  double min_imag() const { return *std::min_element(WI.begin(), WI.end()); }
  double max_imag() const { return *std::max_element(WI.begin(), WI.end()); }
  double min_mag() const { return *std::min_element(WM.begin(), WM.end()); }
  double max_mag() const { return *std::max_element(WM.begin(), WM.end()); }
  double cond_number() const { return max_mag() / min_mag(); }
};
template <typename T, int M, typename PreCond = DevicePrecond<T, M, 1>>
Eigenvalues arnoldi_eigenvalues(const BlockSp::BlockSp<T, M>& A, int iters = 30, const PreCond* preCond = nullptr,
                                bool printEigInfo = false, bool printEigVals = false, bool harmonic_Ritz = false) {
  DeviceMatrix dA(A, M);
  // a preconditioner carries its own device copy of A; the Arnoldi runs on it
  const bsp_matrix_t mat = preCond ? preCond->matrix()->get() : dA.get();
  const bsp_handle_t h = preCond ? preCond->matrix()->handle() : dA.handle();
  Eigenvalues e;
  e.harmonic_Ritz = harmonic_Ritz;
  e.WR.resize(iters);
  e.WI.resize(iters);
  int n = 0;
  check(bsp_arnoldi_eigenvalues(h, mat, preCond ? preCond->get() : nullptr, iters, harmonic_Ritz, printEigInfo,
                                printEigVals, e.WR.data(), e.WI.data(), &n),
        "bsp_arnoldi_eigenvalues", h);
  e.WR.resize(n);
  e.WI.resize(n);
  for (int i = 0; i < n; ++i) e.WM.push_back(std::sqrt(e.WR[i] * e.WR[i] + e.WI[i] * e.WI[i]));
  return e;
}

}  // namespace blocksp_b200
