// complex_dense.h — small dense complex linear algebra on the host for the
// complex pGMRES (blocksp_solvers.hpp:156-295 and blocksp_deflated_restart.hpp:
// 38-269 with T = std::complex<double>): Householder least squares (gels),
// an LU solve (getrf / getrs), the complex Schur form (gehrd + hseqr, i.e.
// gees) with the reordering of selected eigenvalues to the front (trsen), and
// the deflated-restart algebra built on them.  Plain C++: the tests build it
// for the host on its own.
#pragma once
#include <algorithm>
#include <cmath>
#include <complex>
#include <limits>
#include <vector>

namespace bsp {
namespace cd {

using Cx = std::complex<double>;
constexpr double kEpsC = std::numeric_limits<double>::epsilon();

// Row-major dense complex matrix.
struct CMat {
  int r = 0, c = 0;
  std::vector<Cx> a;
  CMat() = default;
  CMat(int rr, int cc) : r(rr), c(cc), a((size_t)rr * cc, Cx(0.0)) {}
  Cx& operator()(int i, int j) { return a[(size_t)i * c + j]; }
  const Cx& operator()(int i, int j) const { return a[(size_t)i * c + j]; }
};

// Givens rotation G = [[cs, sn], [-conj(sn), cs]] (cs real) with
// G [x; y] = [r; 0].
struct Rot {
  double cs;
  Cx sn;
};
inline Rot givens(Cx x, Cx y) {
  const double ay = std::abs(y);
  if (ay == 0.0) return {1.0, Cx(0.0)};
  const double ax = std::abs(x);
  if (ax == 0.0) return {0.0, std::conj(y) / ay};
  const double nrm = std::hypot(ax, ay);
  return {ax / nrm, (x / ax) * std::conj(y) / nrm};
}
// rows p, p+1 of T, columns j0 .. T.c-1: T <- G T
inline void rot_rows(CMat& T, int p, int j0, const Rot& g) {
  for (int j = j0; j < T.c; ++j) {
    const Cx a = T(p, j), b = T(p + 1, j);
    T(p, j) = g.cs * a + g.sn * b;
    T(p + 1, j) = -std::conj(g.sn) * a + g.cs * b;
  }
}
// columns p, p+1 of M, rows 0 .. i1-1: M <- M G^H
inline void rot_cols(CMat& M, int p, int i1, const Rot& g) {
  for (int i = 0; i < i1; ++i) {
    const Cx a = M(i, p), b = M(i, p + 1);
    M(i, p) = g.cs * a + std::conj(g.sn) * b;
    M(i, p + 1) = -g.sn * a + g.cs * b;
  }
}

// min ||rhs - H y||_2 for H m x n (m >= n, full column rank) by Householder QR:
// the least-squares solution gels computes (blocksp_solvers.hpp:199, 224).
inline std::vector<Cx> lstsq(const CMat& H, std::vector<Cx> rhs) {
  CMat R = H;
  const int m = R.r, n = R.c;
  for (int j = 0; j < n; ++j) {
    double nx = 0.0;
    for (int i = j; i < m; ++i) nx += std::norm(R(i, j));
    nx = std::sqrt(nx);
    if (nx == 0.0) continue;
    const Cx x0 = R(j, j);
    const Cx ph = std::abs(x0) > 0.0 ? x0 / std::abs(x0) : Cx(1.0);
    const Cx alpha = -ph * nx;
    std::vector<Cx> v(m - j);
    for (int i = j; i < m; ++i) v[i - j] = R(i, j);
    v[0] -= alpha;
    double vn = 0.0;
    for (const Cx& t : v) vn += std::norm(t);
    if (vn == 0.0) continue;
    // R <- (I - 2 v v^H / v^H v) R on rows j.., columns j..; same on rhs
    for (int col = j; col < n; ++col) {
      Cx s = 0.0;
      for (int i = j; i < m; ++i) s += std::conj(v[i - j]) * R(i, col);
      s *= 2.0 / vn;
      for (int i = j; i < m; ++i) R(i, col) -= s * v[i - j];
    }
    Cx s = 0.0;
    for (int i = j; i < m; ++i) s += std::conj(v[i - j]) * rhs[i];
    s *= 2.0 / vn;
    for (int i = j; i < m; ++i) rhs[i] -= s * v[i - j];
  }
  std::vector<Cx> y(n);
  for (int i = n - 1; i >= 0; --i) {
    Cx s = rhs[i];
    for (int j = i + 1; j < n; ++j) s -= R(i, j) * y[j];
    y[i] = s / R(i, i);
  }
  return y;
}

// Solve M w = e for a square complex M by Gaussian elimination with partial
// pivoting (LUFactor_Arr::invmul, getrf/getrs).
inline std::vector<Cx> lu_solve(CMat M, std::vector<Cx> w) {
  const int n = M.r;
  for (int k = 0; k < n; ++k) {
    int p = k;
    for (int i = k + 1; i < n; ++i)
      if (std::abs(M(i, k)) > std::abs(M(p, k))) p = i;
    if (p != k) {
      for (int j = 0; j < n; ++j) std::swap(M(k, j), M(p, j));
      std::swap(w[k], w[p]);
    }
    for (int i = k + 1; i < n; ++i) {
      const Cx l = M(i, k) / M(k, k);
      for (int j = k + 1; j < n; ++j) M(i, j) -= l * M(k, j);
      w[i] -= l * w[k];
    }
  }
  for (int i = n - 1; i >= 0; --i) {
    Cx s = w[i];
    for (int j = i + 1; j < n; ++j) s -= M(i, j) * w[j];
    w[i] = s / M(i, i);
  }
  return w;
}

// Complex Schur form of an upper Hessenberg T: T <- Z^H T Z upper triangular,
// Z unitary (accumulated into Z).  Implicit single-shift QR sweeps with the
// Wilkinson shift of the trailing 2 x 2 block and deflation of negligible
// subdiagonals; an exceptional shift every 10 sweeps without deflation.
// Returns false if it did not converge in 60 n sweeps.
inline bool schur_hessenberg(CMat& T, CMat& Z) {
  const int n = T.r;
  int hi = n - 1, its = 0, total = 0;
  while (hi > 0) {
    int l = hi;
    for (; l > 0; --l) {
      const double s = std::abs(T(l - 1, l - 1)) + std::abs(T(l, l));
      if (std::abs(T(l, l - 1)) <= kEpsC * (s > 0.0 ? s : 1.0)) break;
    }
    if (l == hi) {
      T(hi, hi - 1) = 0.0;
      --hi;
      its = 0;
      continue;
    }
    if (++total > 60 * n) return false;
    ++its;
    Cx mu;
    if (its % 10 == 0) {
      mu = T(hi, hi) + std::abs(T(hi, hi - 1));
    } else {
      const Cx a = T(hi - 1, hi - 1), b = T(hi - 1, hi), c = T(hi, hi - 1), d = T(hi, hi);
      const Cx half = 0.5 * (a - d);
      const Cx disc = std::sqrt(half * half + b * c);
      const Cx m1 = 0.5 * (a + d) + disc, m2 = 0.5 * (a + d) - disc;
      mu = std::abs(m1 - d) < std::abs(m2 - d) ? m1 : m2;
    }
    Cx x = T(l, l) - mu, y = T(l + 1, l);
    for (int k = l; k < hi; ++k) {
      const Rot g = givens(x, y);
      rot_rows(T, k, k > l ? k - 1 : l, g);
      rot_cols(T, k, std::min(k + 3, hi + 1), g);
      rot_cols(Z, k, Z.r, g);
      if (k > l) T(k + 1, k - 1) = 0.0;
      if (k + 1 < hi) {
        x = T(k + 1, k);
        y = T(k + 2, k);
      }
    }
  }
  return true;
}

// Reduce a square T to upper Hessenberg form by Householder reflections,
// T <- P^H T P, Z <- Z P (gehrd's reduction).
inline void hessenberg_reduce(CMat& T, CMat& Z) {
  const int n = T.r;
  for (int j = 0; j + 2 < n; ++j) {
    double nx = 0.0;
    for (int i = j + 1; i < n; ++i) nx += std::norm(T(i, j));
    nx = std::sqrt(nx);
    if (nx == 0.0) continue;
    const Cx x0 = T(j + 1, j);
    const Cx ph = std::abs(x0) > 0.0 ? x0 / std::abs(x0) : Cx(1.0);
    std::vector<Cx> v(n - j - 1);
    for (int i = j + 1; i < n; ++i) v[i - j - 1] = T(i, j);
    v[0] += ph * nx;
    double vn = 0.0;
    for (const Cx& t : v) vn += std::norm(t);
    if (vn == 0.0) continue;
    // T <- (I - 2 v v^H / v^H v) T on rows j+1..
    for (int col = 0; col < n; ++col) {
      Cx s = 0.0;
      for (int i = j + 1; i < n; ++i) s += std::conj(v[i - j - 1]) * T(i, col);
      s *= 2.0 / vn;
      for (int i = j + 1; i < n; ++i) T(i, col) -= s * v[i - j - 1];
    }
    // T <- T (I - 2 v v^H / v^H v) on columns j+1..; Z likewise
    for (CMat* M : {&T, &Z})
      for (int row = 0; row < M->r; ++row) {
        Cx s = 0.0;
        for (int i = j + 1; i < n; ++i) s += (*M)(row, i) * v[i - j - 1];
        s *= 2.0 / vn;
        for (int i = j + 1; i < n; ++i) (*M)(row, i) -= s * std::conj(v[i - j - 1]);
      }
    for (int i = j + 2; i < n; ++i) T(i, j) = 0.0;
  }
}

// Complex Schur form of a square T (T <- Z^H T Z, Z accumulated).
inline bool schur(CMat& T, CMat& Z) {
  hessenberg_reduce(T, Z);
  return schur_hessenberg(T, Z);
}

// Swap the adjacent diagonal entries p, p+1 of the upper triangular T
// (ztrexc's 1 x 1 exchange): a rotation whose adjoint's first column is the
// eigenvector of T(p+1, p+1) in the leading 2 x 2 block.
inline void schur_swap(CMat& T, CMat& Z, int p) {
  const Cx t11 = T(p, p), t22 = T(p + 1, p + 1);
  const Rot g = givens(T(p, p + 1), t22 - t11);
  rot_rows(T, p, p, g);
  rot_cols(T, p, p + 2, g);
  rot_cols(Z, p, Z.r, g);
  T(p + 1, p) = 0.0;
  T(p, p) = t22;
  T(p + 1, p + 1) = t11;
}

// trsen: move the selected eigenvalues to the leading positions, keeping
// their relative order; returns how many were selected.
inline int schur_reorder(CMat& T, CMat& Z, std::vector<int> select) {
  const int n = T.r;
  int ks = 0;
  for (int k = 0; k < n; ++k) {
    if (!select[k]) continue;
    for (int p = k - 1; p >= ks; --p) {
      schur_swap(T, Z, p);
      std::swap(select[p], select[p + 1]);
    }
    ++ks;
  }
  return ks;
}

// deflated_restart (blocksp_deflated_restart.hpp:38-269), complex branch, on
// the host part: given H ((n+1) x n) and res_vec, returns P_{k+1}
// ((n+1) x (k+1)), the new H = P_{k+1}^H H P_k, the new c_r = P_{k+1}^H res_vec
// and the effective k.  k > 0 and k <= n on entry.
inline int deflate_complex(const CMat& H, const std::vector<Cx>& res_vec, int k, CMat& Pk1, CMat& Hnew,
                    std::vector<Cx>& c_r) {
  const int n = H.c;
  // (1) H_tilde = H_n + |h_mn|^2 H_n^-H e_n e_n^T
  CMat Hn(n, n);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) Hn(i, j) = H(i, j);
  const Cx h_mn = H(n, n - 1);
  CMat HnH(n, n);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) HnH(i, j) = std::conj(Hn(j, i));
  std::vector<Cx> e(n, Cx(0.0));
  e[n - 1] = 1.0;
  const std::vector<Cx> w = lu_solve(HnH, e);
  const Cx scale = std::conj(h_mn) * h_mn;
  for (int i = 0; i < n; ++i) Hn(i, n - 1) += scale * w[i];
  // (2) complex Schur form, the k smallest |theta| first
  CMat Z(n, n);
  for (int i = 0; i < n; ++i) Z(i, i) = 1.0;
  if (!schur(Hn, Z)) return 3;  // the Schur iteration did not converge
  std::vector<int> perm(n);
  for (int i = 0; i < n; ++i) perm[i] = i;
  std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) { return std::abs(Hn(a, a)) < std::abs(Hn(b, b)); });
  std::vector<int> select(n, 0);
  for (int i = 0; i < k; ++i) select[perm[i]] = 1;
  k = schur_reorder(Hn, Z, select);
  // (3) P_k = the first k Schur vectors, orthonormalised (geqrf + ungqr keep
  // their span; Gram-Schmidt here)
  CMat Pk(n, k);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < k; ++j) Pk(i, j) = Z(i, j);
  for (int j = 0; j < k; ++j) {
    for (int pass = 0; pass < 2; ++pass)
      for (int q = 0; q < j; ++q) {
        Cx d = 0.0;
        for (int i = 0; i < n; ++i) d += std::conj(Pk(i, q)) * Pk(i, j);
        for (int i = 0; i < n; ++i) Pk(i, j) -= d * Pk(i, q);
      }
    double nr = 0.0;
    for (int i = 0; i < n; ++i) nr += std::norm(Pk(i, j));
    nr = std::sqrt(nr);
    for (int i = 0; i < n; ++i) Pk(i, j) /= nr;
  }
  // (4) P_{k+1}: P_k over a zero row, then res_vec orthogonalised against it
  Pk1 = CMat(n + 1, k + 1);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < k; ++j) Pk1(i, j) = Pk(i, j);
  for (int i = 0; i < n + 1; ++i) Pk1(i, k) = res_vec[i];
  for (int q = 0; q < k; ++q) {
    Cx d = 0.0;
    for (int j = 0; j < n + 1; ++j) d += std::conj(Pk1(j, q)) * Pk1(j, k);
    for (int j = 0; j < n + 1; ++j) Pk1(j, k) -= d * Pk1(j, q);
  }
  Cx nrm = 0.0;
  for (int j = 0; j < n + 1; ++j) nrm += std::conj(Pk1(j, k)) * Pk1(j, k);
  nrm = std::sqrt(nrm);
  for (int j = 0; j < n + 1; ++j) Pk1(j, k) /= nrm;
  // (5) c_r = P_{k+1}^H res_vec
  c_r.assign(k + 1, Cx(0.0));
  for (int i = 0; i < k + 1; ++i)
    for (int j = 0; j < n + 1; ++j) c_r[i] += std::conj(Pk1(j, i)) * res_vec[j];
  // (6) H_new = P_{k+1}^H (H P_k)
  CMat HP(n + 1, k);
  for (int i = 0; i < n + 1; ++i)
    for (int j = 0; j < k; ++j) {
      Cx s = 0.0;
      for (int t = 0; t < n; ++t) s += H(i, t) * Pk(t, j);
      HP(i, j) = s;
    }
  Hnew = CMat(k + 1, k);
  for (int i = 0; i < k + 1; ++i)
    for (int j = 0; j < k; ++j) {
      Cx s = 0.0;
      for (int t = 0; t < n + 1; ++t) s += std::conj(Pk1(t, i)) * HP(t, j);
      Hnew(i, j) = s;
    }
  return 0;
}

// Ritz values of an Arnoldi H ((n+1) x n): the eigenvalues of its square part
// H_n, or with harmonic the harmonic Ritz values, the eigenvalues of
// H_n + |h_mn|^2 H_n^-H e_n e_n^T (Eigenvalues_Arr's complex branch,
// blocksp_dense_solvers.hpp:919-965).  False if the Schur iteration failed.
inline bool ritz_values(const CMat& H, bool harmonic, std::vector<Cx>& ev) {
  const int n = H.c;
  ev.clear();
  if (n < 1 || H.r < n + 1) return false;
  CMat Hs(n, n), HsH(n, n), Z(n, n);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      Hs(i, j) = H(i, j);
      HsH(j, i) = std::conj(H(i, j));
    }
  if (harmonic) {
    std::vector<Cx> e(n, Cx(0.0));
    e[n - 1] = 1.0;
    const std::vector<Cx> w = lu_solve(HsH, e);
    const Cx hmn = H(n, n - 1);
    for (int i = 0; i < n; ++i) Hs(i, n - 1) += std::conj(hmn) * hmn * w[i];
  }
  for (int i = 0; i < n; ++i) Z(i, i) = 1.0;
  if (!schur(Hs, Z)) return false;
  for (int i = 0; i < n; ++i) ev.push_back(Hs(i, i));
  return true;
}

}  // namespace cd
}  // namespace bsp
