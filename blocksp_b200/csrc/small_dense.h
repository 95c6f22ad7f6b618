// small_dense.h — the small dense FP64 work of pGMRES, as host+device code.
//
// Runs on one GPU warp inside the solver (n <= a few hundred), and compiles
// unchanged with a host C++ compiler so it can be unit-tested on the CPU.
// Matrices are row-major with an explicit leading dimension: A(i,j) = A[i*ld+j].
//
// Every team routine takes a team: SoloTeam on the host (one thread),
// WarpTeam on the device (32 lanes).  Scalar control flow (pivot choice,
// shifts, deflation tests) is evaluated identically by every member from
// shared data; loops over independent rows or columns are split across the
// members, with sync() between phases; serial writes to shared arrays are
// made by member 0.
//
// Reference counterparts (BlockSp v1.0):
//   Givens least squares  <- lapack::gels + gemv on a copy of H every
//                             iteration (blocksp_solvers.hpp:192-232)
//   solve_transposed      <- LUFactor_Arr(H_n^T).invmul (deflated_restart.hpp:76-85)
//   real_schur            <- lapack::gees (deflated_restart.hpp:125-127)
//   select_smallest       <- deflated_restart.hpp:129-165 (same rule)
//   invariant_basis       <- lapack::trsen + geqrf/orgqr (deflated_restart.hpp:167-193):
//                            an orthonormal basis of the same invariant subspace,
//                            built from the selected eigenvectors instead of a
//                            Schur reordering (any such basis yields the same
//                            restarted Krylov space).
// Algorithms: Householder reduction to Hessenberg form and the Francis
// double-shift QR iteration (Golub & Van Loan, Matrix Computations, 4th ed.,
// Alg. 7.4.2 and 7.5.1-7.5.2); eigenvectors of a quasi-triangular matrix by
// back substitution; Householder QR (G&VL Alg. 5.2.1).
#pragma once
#include <math.h>

#if defined(__CUDACC__)
#define BSP_HD __host__ __device__
#else
#define BSP_HD
#endif

namespace bsp {
namespace sd {

struct SoloTeam {
  BSP_HD int rank() const { return 0; }
  BSP_HD int size() const { return 1; }
  BSP_HD void sync() const {}
  BSP_HD double sum(double v) const { return v; }
};
#if defined(__CUDACC__)
struct WarpTeam {
  __device__ int rank() const { return threadIdx.x & 31; }
  __device__ int size() const { return 32; }
  __device__ void sync() const { __syncwarp(); }
  // Butterfly sum: every lane adds the same two operands at each stage (in
  // swapped order, which is exact), so all lanes end with identical bits.
  __device__ double sum(double v) const {
    for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
    return v;
  }
};
#endif

BSP_HD inline double dabs(double x) { return x < 0 ? -x : x; }
BSP_HD inline double dsign(double a, double b) { return b >= 0 ? dabs(a) : -dabs(a); }
BSP_HD inline double dhypot(double a, double b) {
  a = dabs(a);
  b = dabs(b);
  const double m = a > b ? a : b, q = a > b ? b : a;
  if (m == 0.0) return 0.0;
  const double r = q / m;
  return m * sqrt(1.0 + r * r);
}

// ------------------------------------------------------------ Givens LS
// Rotation acting on rows (p, p+1):  [c s; -s c] [a; b] = [r; 0].
struct Rot {
  int p;
  double c, s;
};

BSP_HD inline void make_givens(double a, double b, double& c, double& s) {
  if (b == 0.0) {
    c = 1.0;
    s = 0.0;
    return;
  }
  const double r = dhypot(a, b);
  c = a / r;
  s = b / r;
}
BSP_HD inline void apply_rot(const Rot& g, double* v, int stride) {
  const double a = v[g.p * stride], b = v[(g.p + 1) * stride];
  v[g.p * stride] = g.c * a + g.s * b;
  v[(g.p + 1) * stride] = -g.s * a + g.c * b;
}

// Append column j of H (rows 0..last) to the QR factorisation held in R/rots/g.
// R, H: (m_cap+1) x m_cap row-major (ld = m_cap).  Returns |g[j+1]|, the
// least-squares residual norm after the column is added.  (One thread.)
BSP_HD inline double ls_add_column(const double* H, int ld, int j, int last, double* R, Rot* rots,
                                   int& nrot, double* g) {
  for (int i = 0; i <= last; ++i) R[i * ld + j] = H[i * ld + j];
  for (int t = 0; t < nrot; ++t) apply_rot(rots[t], R + j, ld);
  for (int r = last; r > j; --r) {
    Rot q;
    q.p = r - 1;
    make_givens(R[(r - 1) * ld + j], R[r * ld + j], q.c, q.s);
    apply_rot(q, R + j, ld);
    R[r * ld + j] = 0.0;
    apply_rot(q, g, 1);
    rots[nrot++] = q;
  }
  return dabs(g[j + 1]);
}

// y = R(0:n,0:n)^{-1} g(0:n)   (one thread)
BSP_HD inline void back_solve(const double* R, int ld, const double* g, int n, double* y) {
  for (int i = n - 1; i >= 0; --i) {
    double s = g[i];
    for (int t = i + 1; t < n; ++t) s -= R[i * ld + t] * y[t];
    y[i] = s / R[i * ld + i];
  }
}

// ------------------------------------------------------------ LU solve
// Solve A^T w = b in place (A n x n, row-major, ld), partial pivoting.
// work: n*n doubles.  Returns false if singular.
template <class TM>
BSP_HD inline bool solve_transposed(const TM& tm, const double* A, int ld, int n, double* w, double* work,
                                    int* piv) {
  const int r0 = tm.rank(), ns = tm.size();
  for (int e = r0; e < n * n; e += ns) {
    const int i = e / n, j = e % n;
    work[i * n + j] = A[j * ld + i];  // A^T
  }
  tm.sync();
  bool ok = true;
  for (int k = 0; k < n; ++k) {
    int p = k;
    double best = dabs(work[k * n + k]);
    for (int i = k + 1; i < n; ++i)
      if (dabs(work[i * n + k]) > best) {
        best = dabs(work[i * n + k]);
        p = i;
      }
    if (r0 == 0) piv[k] = p;
    if (best == 0.0) {
      ok = false;
      continue;
    }
    tm.sync();
    if (p != k) {
      for (int j = r0; j < n; j += ns) {
        const double t = work[k * n + j];
        work[k * n + j] = work[p * n + j];
        work[p * n + j] = t;
      }
      if (r0 == 0) {
        const double t = w[k];
        w[k] = w[p];
        w[p] = t;
      }
      tm.sync();
    }
    const double pivot = work[k * n + k];
    const double wk = w[k];
    tm.sync();
    for (int i = k + 1 + r0; i < n; i += ns) {
      const double f = work[i * n + k] / pivot;
      work[i * n + k] = f;
      for (int j = k + 1; j < n; ++j) work[i * n + j] -= f * work[k * n + j];
      w[i] -= f * wk;
    }
    tm.sync();
  }
  if (r0 == 0) {
    for (int i = n - 1; i >= 0; --i) {
      double s = w[i];
      for (int j = i + 1; j < n; ++j) s -= work[i * n + j] * w[j];
      w[i] = s / work[i * n + i];
    }
  }
  tm.sync();
  return ok;
}

// ------------------------------------------------------------ Schur
// Householder reduction of A (n x n, ld) to upper Hessenberg form, Z = Q.
// v: n doubles of scratch shared by the team.
template <class TM>
BSP_HD inline void hessenberg(const TM& tm, double* A, int ld, int n, double* Z, int ldz, double* v) {
  const int r0 = tm.rank(), ns = tm.size();
  for (int e = r0; e < n * n; e += ns) {
    const int i = e / n, j = e % n;
    Z[i * ldz + j] = (i == j) ? 1.0 : 0.0;
  }
  tm.sync();
  for (int k = 0; k + 2 < n; ++k) {
    double alpha = 0.0;
    for (int i = k + 1; i < n; ++i) alpha += A[i * ld + k] * A[i * ld + k];
    alpha = sqrt(alpha);
    if (alpha == 0.0) continue;
    const double x0 = A[(k + 1) * ld + k];
    const double beta = -dsign(alpha, x0);
    double vv = (x0 - beta) * (x0 - beta);
    for (int i = k + 2; i < n; ++i) vv += A[i * ld + k] * A[i * ld + k];
    if (vv == 0.0) continue;
    const double tau = 2.0 / vv;
    tm.sync();
    if (r0 == 0)
      for (int i = k + 1; i < n; ++i) v[i] = (i == k + 1) ? x0 - beta : A[i * ld + k];
    tm.sync();
    // A = H A  (columns independent)
    for (int j = r0; j < n; j += ns) {
      double s = 0.0;
      for (int i = k + 1; i < n; ++i) s += v[i] * A[i * ld + j];
      s *= tau;
      for (int i = k + 1; i < n; ++i) A[i * ld + j] -= s * v[i];
    }
    tm.sync();
    // A = A H, Z = Z H  (rows independent)
    for (int i = r0; i < n; i += ns) {
      double s = 0.0;
      for (int j = k + 1; j < n; ++j) s += A[i * ld + j] * v[j];
      s *= tau;
      for (int j = k + 1; j < n; ++j) A[i * ld + j] -= s * v[j];
      double t = 0.0;
      for (int j = k + 1; j < n; ++j) t += Z[i * ldz + j] * v[j];
      t *= tau;
      for (int j = k + 1; j < n; ++j) Z[i * ldz + j] -= t * v[j];
    }
    tm.sync();
    for (int i = k + 2 + r0; i < n; i += ns) A[i * ld + k] = 0.0;
    tm.sync();
  }
}

// Householder vector for x (len 2 or 3): P x = beta e1, u[0] = 1.
BSP_HD inline double house(const double* x, int len, double* u) {
  double sig = 0.0;
  for (int t = 1; t < len; ++t) sig += x[t] * x[t];
  u[0] = 1.0;
  for (int t = 1; t < len; ++t) u[t] = x[t];
  if (sig == 0.0) return 0.0;
  const double mu = sqrt(x[0] * x[0] + sig);
  const double v0 = (x[0] <= 0.0) ? x[0] - mu : -sig / (x[0] + mu);
  const double tau = 2.0 * v0 * v0 / (sig + v0 * v0);
  for (int t = 1; t < len; ++t) u[t] = x[t] / v0;
  return tau;
}

// P = I - tau u u^T on rows r..r+nr-1 (columns c0..c1) from the left, and on
// columns r..r+nr-1 (rows r0..r1) from the right.
template <class TM>
BSP_HD inline void refl_left(const TM& tm, double* H, int ld, int r, int nr, const double* u, double tau,
                             int c0, int c1) {
  for (int j = c0 + tm.rank(); j <= c1; j += tm.size()) {
    double s = 0.0;
    for (int t = 0; t < nr; ++t) s += u[t] * H[(r + t) * ld + j];
    s *= tau;
    for (int t = 0; t < nr; ++t) H[(r + t) * ld + j] -= s * u[t];
  }
}
template <class TM>
BSP_HD inline void refl_right(const TM& tm, double* H, int ld, int r, int nr, const double* u, double tau,
                              int r0, int r1) {
  for (int i = r0 + tm.rank(); i <= r1; i += tm.size()) {
    double s = 0.0;
    for (int t = 0; t < nr; ++t) s += H[i * ld + r + t] * u[t];
    s *= tau;
    for (int t = 0; t < nr; ++t) H[i * ld + r + t] -= s * u[t];
  }
}

// Split a converged 2x2 diagonal block at rows (i, i+1) with real
// eigenvalues into upper-triangular form by a rotation (updates H and Z).
template <class TM>
BSP_HD inline void split_2x2(const TM& tm, double* H, int ld, int n, double* Z, int ldz, int i) {
  const double a = H[i * ld + i], b = H[i * ld + i + 1], c = H[(i + 1) * ld + i],
               d = H[(i + 1) * ld + i + 1];
  const double p = 0.5 * (a - d);
  const double disc = p * p + b * c;
  if (disc < 0.0 || c == 0.0) return;
  const double sq = sqrt(disc);
  const double lam = d + p + dsign(sq, p);  // eigenvalue farther from d: stable
  // eigenvector (lam - d, c) of the 2x2 block
  const double x = lam - d, y = c;
  const double r = dhypot(x, y);
  if (r == 0.0) return;
  const double cs = x / r, sn = y / r;
  tm.sync();
  // H <- G^T H G with G = [cs -sn; sn cs]
  for (int j = tm.rank(); j < n; j += tm.size()) {
    const double h1 = H[i * ld + j], h2 = H[(i + 1) * ld + j];
    H[i * ld + j] = cs * h1 + sn * h2;
    H[(i + 1) * ld + j] = -sn * h1 + cs * h2;
  }
  tm.sync();
  for (int k = tm.rank(); k < n; k += tm.size()) {
    const double h1 = H[k * ld + i], h2 = H[k * ld + i + 1];
    H[k * ld + i] = cs * h1 + sn * h2;
    H[k * ld + i + 1] = -sn * h1 + cs * h2;
    const double z1 = Z[k * ldz + i], z2 = Z[k * ldz + i + 1];
    Z[k * ldz + i] = cs * z1 + sn * z2;
    Z[k * ldz + i + 1] = -sn * z1 + cs * z2;
  }
  tm.sync();
  if (tm.rank() == 0) H[(i + 1) * ld + i] = 0.0;
  tm.sync();
}

// Real Schur form of the Hessenberg matrix H (in place) by the Francis
// double-shift QR iteration; Z accumulates the transformations (Z_in * Q).
// Returns false if the iteration did not converge.
template <class TM>
BSP_HD inline bool francis_qr(const TM& tm, double* H, int ld, int n, double* Z, int ldz) {
  const double eps = 2.220446049250313e-16;
  const int r0 = tm.rank();
  int hi = n - 1;
  int iter = 0;
  const int max_iter = 60 * n;
  int total = 0;
  while (hi >= 0) {
    if (++total > max_iter) return false;
    // find the start lo of the unreduced block ending at hi
    int lo = hi;
    bool zeroed = false;
    while (lo > 0) {
      const double s = dabs(H[(lo - 1) * ld + lo - 1]) + dabs(H[lo * ld + lo]);
      const double tst = s == 0.0 ? 1.0 : s;
      if (dabs(H[lo * ld + lo - 1]) <= eps * tst) {
        zeroed = true;
        break;
      }
      --lo;
    }
    tm.sync();
    if (zeroed && r0 == 0) H[lo * ld + lo - 1] = 0.0;
    tm.sync();
    if (lo == hi) {  // 1x1 block converged
      --hi;
      iter = 0;
      continue;
    }
    if (lo == hi - 1) {  // 2x2 block converged
      split_2x2(tm, H, ld, n, Z, ldz, hi - 1);
      hi -= 2;
      iter = 0;
      continue;
    }
    ++iter;
    // shifts: eigenvalues of the trailing 2x2 (exceptional shifts every 10 its)
    double s, t;
    if (iter % 10 == 0) {
      const double w = dabs(H[hi * ld + hi - 1]) + dabs(H[(hi - 1) * ld + hi - 2]);
      s = 1.5 * w + H[hi * ld + hi];
      t = w * w;
    } else {
      const double a = H[(hi - 1) * ld + hi - 1], b = H[(hi - 1) * ld + hi],
                   c = H[hi * ld + hi - 1], d = H[hi * ld + hi];
      s = a + d;
      t = a * d - b * c;
    }
    // first column of (H - s1 I)(H - s2 I)
    const double h00 = H[lo * ld + lo], h01 = H[lo * ld + lo + 1], h10 = H[(lo + 1) * ld + lo],
                 h11 = H[(lo + 1) * ld + lo + 1], h21 = H[(lo + 2) * ld + lo + 1];
    double x[3];
    x[0] = h00 * h00 + h01 * h10 - s * h00 + t;
    x[1] = h10 * (h00 + h11 - s);
    x[2] = h10 * h21;
    for (int k = lo; k <= hi - 2; ++k) {
      double u[3];
      const double tau = house(x, 3, u);
      tm.sync();
      if (tau != 0.0) {
        const int c0 = k > lo ? k - 1 : lo;
        refl_left(tm, H, ld, k, 3, u, tau, c0, n - 1);
        tm.sync();
        const int r1 = (k + 3 < hi) ? k + 3 : hi;
        refl_right(tm, H, ld, k, 3, u, tau, 0, r1);
        refl_right(tm, Z, ldz, k, 3, u, tau, 0, n - 1);
        tm.sync();
      }
      if (k > lo && r0 == 0) {
        H[(k + 1) * ld + k - 1] = 0.0;
        H[(k + 2) * ld + k - 1] = 0.0;
      }
      tm.sync();
      x[0] = H[(k + 1) * ld + k];
      x[1] = H[(k + 2) * ld + k];
      if (k < hi - 2) x[2] = H[(k + 3) * ld + k];
    }
    {
      double u[3];
      const int k = hi - 1;
      const double tau = house(x, 2, u);
      tm.sync();
      if (tau != 0.0) {
        refl_left(tm, H, ld, k, 2, u, tau, k - 1, n - 1);
        tm.sync();
        refl_right(tm, H, ld, k, 2, u, tau, 0, hi);
        refl_right(tm, Z, ldz, k, 2, u, tau, 0, n - 1);
        tm.sync();
      }
      if (r0 == 0) H[hi * ld + hi - 2] = 0.0;
      tm.sync();
    }
  }
  return true;
}

// Eigenvalues of a quasi-triangular T: 1x1 blocks real, 2x2 blocks complex
// pairs.  (One thread.)
BSP_HD inline void schur_eigs(const double* T, int ld, int n, double* wr, double* wi) {
  int i = 0;
  while (i < n) {
    if (i + 1 < n && T[(i + 1) * ld + i] != 0.0) {
      const double a = T[i * ld + i], b = T[i * ld + i + 1], c = T[(i + 1) * ld + i],
                   d = T[(i + 1) * ld + i + 1];
      const double p = 0.5 * (a - d);
      const double disc = p * p + b * c;  // < 0 after split_2x2
      const double im = sqrt(dabs(disc));
      wr[i] = wr[i + 1] = d + p;
      wi[i] = im;
      wi[i + 1] = -im;
      i += 2;
    } else {
      wr[i] = T[i * ld + i];
      wi[i] = 0.0;
      i += 1;
    }
  }
}

// Selection rule of deflated_restart.hpp:129-165: indices sorted by |theta|
// (stable insertion sort, ties keep index order), take the k smallest, and
// complete a complex pair with its conjugate.  Returns the count (sdim).
// (One thread.)
BSP_HD inline int select_smallest(const double* wr, const double* wi, int n, int k, double zero_thresh,
                                  int* perm, int* select) {
  for (int i = 0; i < n; ++i) {
    perm[i] = i;
    select[i] = 0;
  }
  for (int i = 1; i < n; ++i) {
    const int v = perm[i];
    const double mv = sqrt(wr[v] * wr[v] + wi[v] * wi[v]);
    int j = i - 1;
    while (j >= 0) {
      const int u = perm[j];
      const double mu = sqrt(wr[u] * wr[u] + wi[u] * wi[u]);
      if (mu > mv) {
        perm[j + 1] = u;
        --j;
      } else {
        break;
      }
    }
    perm[j + 1] = v;
  }
  int cnt = 0;
  for (int i = 0; i < n && cnt < k; ++i) {
    const int ip = perm[i];
    if (select[ip]) continue;
    select[ip] = 1;
    cnt++;
    if (dabs(wi[ip]) > zero_thresh) {
      for (int j = 0; j < n; ++j) {
        if (j != ip && dabs(wr[j] - wr[ip]) < zero_thresh && dabs(wi[j] + wi[ip]) < zero_thresh) {
          if (!select[j]) {
            select[j] = 1;
            cnt++;
          }
          break;
        }
      }
    }
  }
  return cnt;
}

// Householder QR of P (n x k, ld): overwrite P with the thin Q.  work: n*k + n.
template <class TM>
BSP_HD inline void orthonormalize(const TM& tm, double* P, int ld, int n, int k, double* work) {
  const int r0 = tm.rank(), ns = tm.size();
  double* Rf = work;  // copy holding the reflectors (n x k)
  double* taus = work + n * k;
  for (int e = r0; e < n * k; e += ns) {
    const int i = e / k, j = e % k;
    Rf[i * k + j] = P[i * ld + j];
  }
  tm.sync();
  for (int j = 0; j < k; ++j) {
    double alpha = 0.0;
    for (int i = j; i < n; ++i) alpha += Rf[i * k + j] * Rf[i * k + j];
    alpha = sqrt(alpha);
    const double x0 = Rf[j * k + j];
    const double beta = -dsign(alpha, x0);
    const double v0 = x0 - beta;
    const bool skip = (alpha == 0.0 || v0 == 0.0);
    const double tau = skip ? 0.0 : (beta - x0) / beta;
    tm.sync();
    if (r0 == 0) {
      taus[j] = tau;
      if (!skip) {
        for (int i = j + 1; i < n; ++i) Rf[i * k + j] /= v0;
        Rf[j * k + j] = beta;
      }
    }
    tm.sync();
    if (skip) continue;
    // v = (1, Rf[j+1:, j]); apply H_j to the remaining columns
    for (int c = j + 1 + r0; c < k; c += ns) {
      double s = Rf[j * k + c];
      for (int i = j + 1; i < n; ++i) s += Rf[i * k + j] * Rf[i * k + c];
      s *= tau;
      Rf[j * k + c] -= s;
      for (int i = j + 1; i < n; ++i) Rf[i * k + c] -= s * Rf[i * k + j];
    }
    tm.sync();
  }
  // form Q = H_0 ... H_{k-1} [I_k; 0]
  for (int e = r0; e < n * k; e += ns) {
    const int i = e / k, j = e % k;
    P[i * ld + j] = (i == j) ? 1.0 : 0.0;
  }
  tm.sync();
  for (int j = k - 1; j >= 0; --j) {
    const double tau = taus[j];
    if (tau == 0.0) continue;
    for (int c = j + r0; c < k; c += ns) {
      double s = P[j * ld + c];
      for (int i = j + 1; i < n; ++i) s += Rf[i * k + j] * P[i * ld + c];
      s *= tau;
      P[j * ld + c] -= s;
      for (int i = j + 1; i < n; ++i) P[i * ld + c] -= s * Rf[i * k + j];
    }
    tm.sync();
  }
}

// Eigenvector y (real part yr, imaginary part yi) of the quasi-triangular T
// for the eigenvalue of the 1x1 block at p (complex == false) or of the 2x2
// block at (p, p+1) (complex == true).  One thread.
BSP_HD inline void quasi_tri_eigvec(const double* T, int ld, int n, int p, bool complex, double lr, double li,
                                    double smin, double* yr, double* yi) {
  for (int t = 0; t < n; ++t) {
    yr[t] = 0.0;
    yi[t] = 0.0;
  }
  if (!complex) {
    yr[p] = 1.0;
    int r = p - 1;
    while (r >= 0) {
      const bool blk2 = r >= 1 && T[r * ld + r - 1] != 0.0;
      if (!blk2) {
        double s = 0.0;
        for (int t = r + 1; t <= p; ++t) s -= T[r * ld + t] * yr[t];
        double den = T[r * ld + r] - lr;
        if (dabs(den) < smin) den = smin;
        yr[r] = s / den;
        r -= 1;
      } else {
        double s0 = 0.0, s1 = 0.0;
        for (int t = r + 1; t <= p; ++t) {
          s0 -= T[(r - 1) * ld + t] * yr[t];
          s1 -= T[r * ld + t] * yr[t];
        }
        const double a = T[(r - 1) * ld + r - 1] - lr, b = T[(r - 1) * ld + r], c = T[r * ld + r - 1],
                     d = T[r * ld + r] - lr;
        double det = a * d - b * c;
        if (dabs(det) < smin) det = smin;
        yr[r - 1] = (d * s0 - b * s1) / det;
        yr[r] = (-c * s0 + a * s1) / det;
        r -= 2;
      }
    }
    return;
  }
  // (t00 - lam) u0 + t01 u1 = 0  ->  u = (t01, lam - t00)
  const double t00 = T[p * ld + p], t01 = T[p * ld + p + 1];
  yr[p] = t01;
  yr[p + 1] = lr - t00;
  yi[p + 1] = li;
  int r = p - 1;
  while (r >= 0) {
    const bool blk2 = r >= 1 && T[r * ld + r - 1] != 0.0;
    if (!blk2) {
      double sr = 0.0, si = 0.0;
      for (int t = r + 1; t <= p + 1; ++t) {
        sr -= T[r * ld + t] * yr[t];
        si -= T[r * ld + t] * yi[t];
      }
      // divide by (T_rr - lam) = (dr - i li)
      const double dr = T[r * ld + r] - lr, di = -li;
      double den = dr * dr + di * di;
      if (den < smin * smin) den = smin * smin;
      yr[r] = (sr * dr + si * di) / den;
      yi[r] = (si * dr - sr * di) / den;
      r -= 1;
    } else {
      double s0r = 0.0, s0i = 0.0, s1r = 0.0, s1i = 0.0;
      for (int t = r + 1; t <= p + 1; ++t) {
        s0r -= T[(r - 1) * ld + t] * yr[t];
        s0i -= T[(r - 1) * ld + t] * yi[t];
        s1r -= T[r * ld + t] * yr[t];
        s1i -= T[r * ld + t] * yi[t];
      }
      // [a b; c d] with a = T00 - lam, d = T11 - lam (complex), b, c real
      const double ar = T[(r - 1) * ld + r - 1] - lr, ai = -li, b = T[(r - 1) * ld + r],
                   c = T[r * ld + r - 1], dr = T[r * ld + r] - lr, di = -li;
      double detr = ar * dr - ai * di - b * c, deti = ar * di + ai * dr;
      double dd = detr * detr + deti * deti;
      if (dd < smin * smin) {
        detr = smin;
        deti = 0.0;
        dd = smin * smin;
      }
      // x0 = (d s0 - b s1)/det, x1 = (-c s0 + a s1)/det
      const double n0r = dr * s0r - di * s0i - b * s1r, n0i = dr * s0i + di * s0r - b * s1i;
      const double n1r = -c * s0r + ar * s1r - ai * s1i, n1i = -c * s0i + ar * s1i + ai * s1r;
      yr[r - 1] = (n0r * detr + n0i * deti) / dd;
      yi[r - 1] = (n0i * detr - n0r * deti) / dd;
      yr[r] = (n1r * detr + n1i * deti) / dd;
      yi[r] = (n1i * detr - n1r * deti) / dd;
      r -= 2;
    }
  }
}

// Basis of the invariant subspace of T (quasi-triangular, from francis_qr)
// belonging to the selected eigenvalues, mapped through Z and orthonormalised.
// Output P (n x k_out, ld = ldp).  work: >= n*n + 4n doubles.
template <class TM>
BSP_HD inline int invariant_basis(const TM& tm, const double* T, int ld, int n, const double* Z, int ldz,
                                  const double* wr, const double* wi, const int* select, double* P,
                                  int ldp, double* work) {
  const double eps = 2.220446049250313e-16;
  const int r0 = tm.rank(), ns = tm.size();
  double tnorm = 0.0;
  for (int i = 0; i < n; ++i)
    for (int j = i > 0 ? i - 1 : 0; j < n; ++j) tnorm = fmax(tnorm, dabs(T[i * ld + j]));
  const double smin = fmax(eps * tnorm, 1e-300);
  double* yr = work;
  double* yi = work + n;
  int kout = 0;
  int i = 0;
  while (i < n) {
    const bool pair = (i + 1 < n) && T[(i + 1) * ld + i] != 0.0;
    const int p = i;
    const bool take = pair ? (select[p] || select[p + 1]) : select[p] != 0;
    if (take) {
      tm.sync();
      if (r0 == 0) quasi_tri_eigvec(T, ld, n, p, pair, wr[p], pair ? dabs(wi[p]) : 0.0, smin, yr, yi);
      tm.sync();
      const int hi = pair ? p + 1 : p;
      for (int t = r0; t < n; t += ns) {
        double s0 = 0.0, s1 = 0.0;
        for (int q = 0; q <= hi; ++q) {
          s0 += Z[t * ldz + q] * yr[q];
          s1 += Z[t * ldz + q] * yi[q];
        }
        P[t * ldp + kout] = s0;
        if (pair) P[t * ldp + kout + 1] = s1;
      }
      kout += pair ? 2 : 1;
    }
    i += pair ? 2 : 1;
  }
  tm.sync();
  if (kout > 0) orthonormalize(tm, P, ldp, n, kout, work + 2 * n);
  return kout;
}

}  // namespace sd
}  // namespace bsp
