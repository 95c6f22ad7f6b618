// Host build of blocksp_b200/csrc/small_dense.h for CPU unit tests (ctypes).
#include <vector>
#include "../../blocksp_b200/csrc/small_dense.h"

using namespace bsp::sd;

extern "C" {

// Real Schur form: A (n x n row-major) -> T, Z with A = Z T Z^T; eigenvalues.
int sd_schur(const double* A, int n, double* T, double* Z, double* wr, double* wi) {
  std::vector<double> v(n + 1);
  for (int i = 0; i < n * n; ++i) T[i] = A[i];
  hessenberg(SoloTeam{}, T, n, n, Z, n, v.data());
  const bool ok = francis_qr(SoloTeam{}, T, n, n, Z, n);
  schur_eigs(T, n, n, wr, wi);
  return ok ? 1 : 0;
}

// Orthonormal basis of the invariant subspace of the k smallest |eig| of A.
int sd_invariant(const double* A, int n, int k, double zero_thresh, double* P, int* keff) {
  std::vector<double> T(n * n), Z(n * n), wr(n), wi(n), work(n * n + 8 * n + 32), v(n + 1);
  std::vector<int> perm(n), sel(n);
  for (int i = 0; i < n * n; ++i) T[i] = A[i];
  hessenberg(SoloTeam{}, T.data(), n, n, Z.data(), n, v.data());
  const bool ok = francis_qr(SoloTeam{}, T.data(), n, n, Z.data(), n);
  schur_eigs(T.data(), n, n, wr.data(), wi.data());
  select_smallest(wr.data(), wi.data(), n, k, zero_thresh, perm.data(), sel.data());
  *keff = invariant_basis(SoloTeam{}, T.data(), n, n, Z.data(), n, wr.data(), wi.data(), sel.data(), P, n,
                          work.data());
  return ok ? 1 : 0;
}

// Givens least squares over the first ncols columns of H ((m+1) x m, ld m)
// with right-hand side rhs (m+1); returns residual norm, y in y.
double sd_lstsq(const double* H, int m, int ncols, int last_row_dense, const double* rhs, double* y) {
  std::vector<double> R((m + 1) * m), g(rhs, rhs + m + 1);
  std::vector<Rot> rots((m + 1) * (m + 2) / 2 + m + 8);
  int nrot = 0;
  double res = 0;
  for (int j = 0; j < ncols; ++j) {
    const int last = j < last_row_dense ? last_row_dense : j + 1;
    res = ls_add_column(H, m, j, last, R.data(), rots.data(), nrot, g.data());
  }
  back_solve(R.data(), m, g.data(), ncols, y);
  return res;
}

int sd_solve_transposed(const double* A, int n, double* w) {
  std::vector<double> work(n * n);
  std::vector<int> piv(n);
  return solve_transposed(SoloTeam{}, A, n, n, w, work.data(), piv.data()) ? 1 : 0;
}
}
