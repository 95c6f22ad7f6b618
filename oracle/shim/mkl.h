// oracle/shim/mkl.h — the Intel MKL C interface subset BlockSp v1.0 calls.
//
// TEST INFRASTRUCTURE ONLY.  MKL is not installed in this image.  This header
// declares the LAPACKE / CBLAS entry points that blocksp_lapack.hpp calls and
// forwards each one to the same routine in scipy's bundled OpenBLAS, which
// exports the standard LAPACKE and CBLAS C API with a "scipy_" prefix and
// 32-bit integers.  mkl_?imatcopy / mkl_?omatcopy (MKL extensions) are
// implemented here from their documented semantics.  Prototypes follow the
// public LAPACKE / CBLAS documentation.
#ifndef BSP_ORACLE_MKL_SHIM_H
#define BSP_ORACLE_MKL_SHIM_H

#include <complex>
#include <cstddef>
#include <vector>

typedef int MKL_INT;
typedef int lapack_int;
typedef int lapack_logical;
typedef std::complex<float> MKL_Complex8;
typedef std::complex<double> MKL_Complex16;

#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102

typedef enum { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_LAYOUT;
typedef CBLAS_LAYOUT CBLAS_ORDER;
typedef enum { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 } CBLAS_TRANSPOSE;

typedef lapack_logical (*LAPACK_S_SELECT2)(const float*, const float*);
typedef lapack_logical (*LAPACK_D_SELECT2)(const double*, const double*);
typedef lapack_logical (*LAPACK_C_SELECT1)(const MKL_Complex8*);
typedef lapack_logical (*LAPACK_Z_SELECT1)(const MKL_Complex16*);

#define BSP_L(x) scipy_LAPACKE_##x
extern "C" {
// ---- CBLAS ----
void scipy_cblas_sgemm(CBLAS_LAYOUT, CBLAS_TRANSPOSE, CBLAS_TRANSPOSE, MKL_INT, MKL_INT, MKL_INT, float,
                       const float*, MKL_INT, const float*, MKL_INT, float, float*, MKL_INT);
void scipy_cblas_dgemm(CBLAS_LAYOUT, CBLAS_TRANSPOSE, CBLAS_TRANSPOSE, MKL_INT, MKL_INT, MKL_INT, double,
                       const double*, MKL_INT, const double*, MKL_INT, double, double*, MKL_INT);
void scipy_cblas_cgemm(CBLAS_LAYOUT, CBLAS_TRANSPOSE, CBLAS_TRANSPOSE, MKL_INT, MKL_INT, MKL_INT, const void*,
                       const void*, MKL_INT, const void*, MKL_INT, const void*, void*, MKL_INT);
void scipy_cblas_zgemm(CBLAS_LAYOUT, CBLAS_TRANSPOSE, CBLAS_TRANSPOSE, MKL_INT, MKL_INT, MKL_INT, const void*,
                       const void*, MKL_INT, const void*, MKL_INT, const void*, void*, MKL_INT);
void scipy_cblas_sgemv(CBLAS_LAYOUT, CBLAS_TRANSPOSE, MKL_INT, MKL_INT, float, const float*, MKL_INT,
                       const float*, MKL_INT, float, float*, MKL_INT);
void scipy_cblas_dgemv(CBLAS_LAYOUT, CBLAS_TRANSPOSE, MKL_INT, MKL_INT, double, const double*, MKL_INT,
                       const double*, MKL_INT, double, double*, MKL_INT);
void scipy_cblas_cgemv(CBLAS_LAYOUT, CBLAS_TRANSPOSE, MKL_INT, MKL_INT, const void*, const void*, MKL_INT,
                       const void*, MKL_INT, const void*, void*, MKL_INT);
void scipy_cblas_zgemv(CBLAS_LAYOUT, CBLAS_TRANSPOSE, MKL_INT, MKL_INT, const void*, const void*, MKL_INT,
                       const void*, MKL_INT, const void*, void*, MKL_INT);

// ---- LAPACKE: real ----
#define BSP_REAL_DECLS(p, T)                                                                              \
  lapack_int BSP_L(p##gels)(int, char, lapack_int, lapack_int, lapack_int, T*, lapack_int, T*, lapack_int); \
  lapack_int BSP_L(p##geqrf)(int, lapack_int, lapack_int, T*, lapack_int, T*);                            \
  lapack_int BSP_L(p##orgqr)(int, lapack_int, lapack_int, lapack_int, T*, lapack_int, const T*);          \
  lapack_int BSP_L(p##getrf)(int, lapack_int, lapack_int, T*, lapack_int, lapack_int*);                   \
  lapack_int BSP_L(p##getrs)(int, char, lapack_int, lapack_int, const T*, lapack_int, const lapack_int*,  \
                             T*, lapack_int);                                                              \
  lapack_int BSP_L(p##pptrf)(int, char, lapack_int, T*);                                                  \
  lapack_int BSP_L(p##pptrs)(int, char, lapack_int, lapack_int, const T*, T*, lapack_int);                \
  lapack_int BSP_L(p##potrf)(int, char, lapack_int, T*, lapack_int);                                      \
  lapack_int BSP_L(p##potrs)(int, char, lapack_int, lapack_int, const T*, lapack_int, T*, lapack_int);    \
  lapack_int BSP_L(p##trtrs)(int, char, char, char, lapack_int, lapack_int, const T*, lapack_int, T*,     \
                             lapack_int);                                                                  \
  lapack_int BSP_L(p##sytrd)(int, char, lapack_int, T*, lapack_int, T*, T*, T*);                          \
  lapack_int BSP_L(p##sterf)(lapack_int, T*, T*);                                                         \
  lapack_int BSP_L(p##syevr)(int, char, char, char, lapack_int, T*, lapack_int, T, T, lapack_int,         \
                             lapack_int, T, lapack_int*, T*, T*, lapack_int, lapack_int*);                \
  lapack_int BSP_L(p##gehrd)(int, lapack_int, lapack_int, lapack_int, T*, lapack_int, T*);                \
  lapack_int BSP_L(p##orghr)(int, lapack_int, lapack_int, lapack_int, T*, lapack_int, const T*);          \
  lapack_int BSP_L(p##hseqr)(int, char, char, lapack_int, lapack_int, lapack_int, T*, lapack_int, T*, T*, \
                             T*, lapack_int);                                                              \
  lapack_int BSP_L(p##trsen)(int, char, char, const lapack_logical*, lapack_int, T*, lapack_int, T*,      \
                             lapack_int, T*, T*, lapack_int*, T*, T*);                                     \
  lapack_int BSP_L(p##ggev)(int, char, char, lapack_int, T*, lapack_int, T*, lapack_int, T*, T*, T*, T*,  \
                            lapack_int, T*, lapack_int);                                                   \
  T BSP_L(p##lange)(int, char, lapack_int, lapack_int, const T*, lapack_int);
BSP_REAL_DECLS(s, float)
BSP_REAL_DECLS(d, double)
#undef BSP_REAL_DECLS
lapack_int scipy_LAPACKE_sgees(int, char, char, LAPACK_S_SELECT2, lapack_int, float*, lapack_int, lapack_int*,
                               float*, float*, float*, lapack_int);
lapack_int scipy_LAPACKE_dgees(int, char, char, LAPACK_D_SELECT2, lapack_int, double*, lapack_int, lapack_int*,
                               double*, double*, double*, lapack_int);

// ---- LAPACKE: complex ----
#define BSP_CPLX_DECLS(p, C, R)                                                                           \
  lapack_int BSP_L(p##gels)(int, char, lapack_int, lapack_int, lapack_int, C*, lapack_int, C*, lapack_int); \
  lapack_int BSP_L(p##geqrf)(int, lapack_int, lapack_int, C*, lapack_int, C*);                            \
  lapack_int BSP_L(p##ungqr)(int, lapack_int, lapack_int, lapack_int, C*, lapack_int, const C*);          \
  lapack_int BSP_L(p##getrf)(int, lapack_int, lapack_int, C*, lapack_int, lapack_int*);                   \
  lapack_int BSP_L(p##getrs)(int, char, lapack_int, lapack_int, const C*, lapack_int, const lapack_int*,  \
                             C*, lapack_int);                                                              \
  lapack_int BSP_L(p##pptrf)(int, char, lapack_int, C*);                                                  \
  lapack_int BSP_L(p##pptrs)(int, char, lapack_int, lapack_int, const C*, C*, lapack_int);                \
  lapack_int BSP_L(p##potrf)(int, char, lapack_int, C*, lapack_int);                                      \
  lapack_int BSP_L(p##potrs)(int, char, lapack_int, lapack_int, const C*, lapack_int, C*, lapack_int);    \
  lapack_int BSP_L(p##trtrs)(int, char, char, char, lapack_int, lapack_int, const C*, lapack_int, C*,     \
                             lapack_int);                                                                  \
  lapack_int BSP_L(p##gehrd)(int, lapack_int, lapack_int, lapack_int, C*, lapack_int, C*);                \
  lapack_int BSP_L(p##unghr)(int, lapack_int, lapack_int, lapack_int, C*, lapack_int, const C*);          \
  lapack_int BSP_L(p##hseqr)(int, char, char, lapack_int, lapack_int, lapack_int, C*, lapack_int, C*, C*, \
                             lapack_int);                                                                  \
  lapack_int BSP_L(p##trsen)(int, char, char, const lapack_logical*, lapack_int, C*, lapack_int, C*,      \
                             lapack_int, C*, lapack_int*, R*, R*);                                         \
  lapack_int BSP_L(p##ggev)(int, char, char, lapack_int, C*, lapack_int, C*, lapack_int, C*, C*, C*,      \
                            lapack_int, C*, lapack_int);                                                   \
  R BSP_L(p##lange)(int, char, lapack_int, lapack_int, const C*, lapack_int);
BSP_CPLX_DECLS(c, MKL_Complex8, float)
BSP_CPLX_DECLS(z, MKL_Complex16, double)
#undef BSP_CPLX_DECLS
lapack_int scipy_LAPACKE_cgees(int, char, char, LAPACK_C_SELECT1, lapack_int, MKL_Complex8*, lapack_int,
                               lapack_int*, MKL_Complex8*, MKL_Complex8*, lapack_int);
lapack_int scipy_LAPACKE_zgees(int, char, char, LAPACK_Z_SELECT1, lapack_int, MKL_Complex16*, lapack_int,
                               lapack_int*, MKL_Complex16*, MKL_Complex16*, lapack_int);
}  // extern "C"
#undef BSP_L

// names used by the reference -> scipy-prefixed symbols
#define cblas_sgemm scipy_cblas_sgemm
#define cblas_dgemm scipy_cblas_dgemm
#define cblas_cgemm scipy_cblas_cgemm
#define cblas_zgemm scipy_cblas_zgemm
#define cblas_sgemv scipy_cblas_sgemv
#define cblas_dgemv scipy_cblas_dgemv
#define cblas_cgemv scipy_cblas_cgemv
#define cblas_zgemv scipy_cblas_zgemv
#define BSP_MAP4(f) \
  BSP_MAP1(s##f) BSP_MAP1(d##f) BSP_MAP1(c##f) BSP_MAP1(z##f)
// (the preprocessor cannot generate #defines; list them)
#define LAPACKE_sgels scipy_LAPACKE_sgels
#define LAPACKE_dgels scipy_LAPACKE_dgels
#define LAPACKE_cgels scipy_LAPACKE_cgels
#define LAPACKE_zgels scipy_LAPACKE_zgels
#define LAPACKE_sgeqrf scipy_LAPACKE_sgeqrf
#define LAPACKE_dgeqrf scipy_LAPACKE_dgeqrf
#define LAPACKE_cgeqrf scipy_LAPACKE_cgeqrf
#define LAPACKE_zgeqrf scipy_LAPACKE_zgeqrf
#define LAPACKE_sorgqr scipy_LAPACKE_sorgqr
#define LAPACKE_dorgqr scipy_LAPACKE_dorgqr
#define LAPACKE_cungqr scipy_LAPACKE_cungqr
#define LAPACKE_zungqr scipy_LAPACKE_zungqr
#define LAPACKE_sgetrf scipy_LAPACKE_sgetrf
#define LAPACKE_dgetrf scipy_LAPACKE_dgetrf
#define LAPACKE_cgetrf scipy_LAPACKE_cgetrf
#define LAPACKE_zgetrf scipy_LAPACKE_zgetrf
#define LAPACKE_sgetrs scipy_LAPACKE_sgetrs
#define LAPACKE_dgetrs scipy_LAPACKE_dgetrs
#define LAPACKE_cgetrs scipy_LAPACKE_cgetrs
#define LAPACKE_zgetrs scipy_LAPACKE_zgetrs
#define LAPACKE_spptrf scipy_LAPACKE_spptrf
#define LAPACKE_dpptrf scipy_LAPACKE_dpptrf
#define LAPACKE_cpptrf scipy_LAPACKE_cpptrf
#define LAPACKE_zpptrf scipy_LAPACKE_zpptrf
#define LAPACKE_spptrs scipy_LAPACKE_spptrs
#define LAPACKE_dpptrs scipy_LAPACKE_dpptrs
#define LAPACKE_cpptrs scipy_LAPACKE_cpptrs
#define LAPACKE_zpptrs scipy_LAPACKE_zpptrs
#define LAPACKE_spotrf scipy_LAPACKE_spotrf
#define LAPACKE_dpotrf scipy_LAPACKE_dpotrf
#define LAPACKE_cpotrf scipy_LAPACKE_cpotrf
#define LAPACKE_zpotrf scipy_LAPACKE_zpotrf
#define LAPACKE_spotrs scipy_LAPACKE_spotrs
#define LAPACKE_dpotrs scipy_LAPACKE_dpotrs
#define LAPACKE_cpotrs scipy_LAPACKE_cpotrs
#define LAPACKE_zpotrs scipy_LAPACKE_zpotrs
#define LAPACKE_strtrs scipy_LAPACKE_strtrs
#define LAPACKE_dtrtrs scipy_LAPACKE_dtrtrs
#define LAPACKE_ctrtrs scipy_LAPACKE_ctrtrs
#define LAPACKE_ztrtrs scipy_LAPACKE_ztrtrs
#define LAPACKE_ssytrd scipy_LAPACKE_ssytrd
#define LAPACKE_dsytrd scipy_LAPACKE_dsytrd
#define LAPACKE_ssterf scipy_LAPACKE_ssterf
#define LAPACKE_dsterf scipy_LAPACKE_dsterf
#define LAPACKE_ssyevr scipy_LAPACKE_ssyevr
#define LAPACKE_dsyevr scipy_LAPACKE_dsyevr
#define LAPACKE_sgehrd scipy_LAPACKE_sgehrd
#define LAPACKE_dgehrd scipy_LAPACKE_dgehrd
#define LAPACKE_cgehrd scipy_LAPACKE_cgehrd
#define LAPACKE_zgehrd scipy_LAPACKE_zgehrd
#define LAPACKE_sorghr scipy_LAPACKE_sorghr
#define LAPACKE_dorghr scipy_LAPACKE_dorghr
#define LAPACKE_cunghr scipy_LAPACKE_cunghr
#define LAPACKE_zunghr scipy_LAPACKE_zunghr
#define LAPACKE_shseqr scipy_LAPACKE_shseqr
#define LAPACKE_dhseqr scipy_LAPACKE_dhseqr
#define LAPACKE_chseqr scipy_LAPACKE_chseqr
#define LAPACKE_zhseqr scipy_LAPACKE_zhseqr
#define LAPACKE_sgees scipy_LAPACKE_sgees
#define LAPACKE_dgees scipy_LAPACKE_dgees
#define LAPACKE_cgees scipy_LAPACKE_cgees
#define LAPACKE_zgees scipy_LAPACKE_zgees
#define LAPACKE_strsen scipy_LAPACKE_strsen
#define LAPACKE_dtrsen scipy_LAPACKE_dtrsen
#define LAPACKE_ctrsen scipy_LAPACKE_ctrsen
#define LAPACKE_ztrsen scipy_LAPACKE_ztrsen
#define LAPACKE_sggev scipy_LAPACKE_sggev
#define LAPACKE_dggev scipy_LAPACKE_dggev
#define LAPACKE_cggev scipy_LAPACKE_cggev
#define LAPACKE_zggev scipy_LAPACKE_zggev
#define LAPACKE_slange scipy_LAPACKE_slange
#define LAPACKE_dlange scipy_LAPACKE_dlange
#define LAPACKE_clange scipy_LAPACKE_clange
#define LAPACKE_zlange scipy_LAPACKE_zlange

// ---- mkl_?imatcopy / mkl_?omatcopy (row-major 'r' and column-major 'c';
//      trans 'n', 't', 'c' (conjugate transpose), 'r' (conjugate)) ----
namespace bsp_mkl_shim {
template <typename T> inline T cj(const T& v) { return v; }
template <typename U> inline std::complex<U> cj(const std::complex<U>& v) { return std::conj(v); }
template <typename T>
inline void omatcopy(char ordering, char trans, size_t rows, size_t cols, T alpha, const T* A, size_t lda,
                     T* B, size_t ldb) {
  const bool row = (ordering == 'r' || ordering == 'R');
  // logical rows x cols source; element (i, j) at A[i*lda + j] (row-major) or A[j*lda + i]
  auto a = [&](size_t i, size_t j) { return row ? A[i * lda + j] : A[j * lda + i]; };
  const char t = (char)(trans | 0x20);
  const bool tr = (t == 't' || t == 'c');
  const bool conj = (t == 'c' || t == 'r');
  for (size_t i = 0; i < rows; ++i)
    for (size_t j = 0; j < cols; ++j) {
      T v = alpha * (conj ? cj(a(i, j)) : a(i, j));
      const size_t bi = tr ? j : i, bj = tr ? i : j;
      if (row) B[bi * ldb + bj] = v;
      else B[bj * ldb + bi] = v;
    }
}
template <typename T>
inline void imatcopy(char ordering, char trans, size_t rows, size_t cols, T alpha, T* AB, size_t lda,
                     size_t ldb) {
  const bool row = (ordering == 'r' || ordering == 'R');
  const size_t n = row ? rows * lda : cols * lda;
  std::vector<T> tmp(AB, AB + n);
  omatcopy(ordering, trans, rows, cols, alpha, tmp.data(), lda, AB, ldb);
}
}  // namespace bsp_mkl_shim

inline void mkl_simatcopy(char o, char t, size_t r, size_t c, float a, float* AB, size_t lda, size_t ldb) {
  bsp_mkl_shim::imatcopy(o, t, r, c, a, AB, lda, ldb);
}
inline void mkl_dimatcopy(char o, char t, size_t r, size_t c, double a, double* AB, size_t lda, size_t ldb) {
  bsp_mkl_shim::imatcopy(o, t, r, c, a, AB, lda, ldb);
}
inline void mkl_cimatcopy(char o, char t, size_t r, size_t c, MKL_Complex8 a, MKL_Complex8* AB, size_t lda,
                          size_t ldb) {
  bsp_mkl_shim::imatcopy(o, t, r, c, a, AB, lda, ldb);
}
inline void mkl_zimatcopy(char o, char t, size_t r, size_t c, MKL_Complex16 a, MKL_Complex16* AB, size_t lda,
                          size_t ldb) {
  bsp_mkl_shim::imatcopy(o, t, r, c, a, AB, lda, ldb);
}
inline void mkl_somatcopy(char o, char t, size_t r, size_t c, float a, const float* A, size_t lda, float* B,
                          size_t ldb) {
  bsp_mkl_shim::omatcopy(o, t, r, c, a, A, lda, B, ldb);
}
inline void mkl_domatcopy(char o, char t, size_t r, size_t c, double a, const double* A, size_t lda,
                          double* B, size_t ldb) {
  bsp_mkl_shim::omatcopy(o, t, r, c, a, A, lda, B, ldb);
}
inline void mkl_comatcopy(char o, char t, size_t r, size_t c, MKL_Complex8 a, const MKL_Complex8* A,
                          size_t lda, MKL_Complex8* B, size_t ldb) {
  bsp_mkl_shim::omatcopy(o, t, r, c, a, A, lda, B, ldb);
}
inline void mkl_zomatcopy(char o, char t, size_t r, size_t c, MKL_Complex16 a, const MKL_Complex16* A,
                          size_t lda, MKL_Complex16* B, size_t ldb) {
  bsp_mkl_shim::omatcopy(o, t, r, c, a, A, lda, B, ldb);
}

#endif
