// Host build of blocksp_b200/csrc/complex_dense.h for the CPU tests
// (tests/test_complex_dense.py): C entry points over interleaved complex
// arrays.
#include <cstring>
#include "../../blocksp_b200/csrc/complex_dense.h"

using namespace bsp::cd;

static CMat load(const double* a, int r, int c) {
  CMat m(r, c);
  std::memcpy(m.a.data(), a, sizeof(double) * 2 * r * c);
  return m;
}
static void store(const CMat& m, double* out) { std::memcpy(out, m.a.data(), sizeof(double) * 2 * m.r * m.c); }

extern "C" {

// A = Z T Z^H with T upper triangular; returns 1 when the iteration converged
int cd_schur(const double* A, int n, double* T, double* Z) {
  CMat t = load(A, n, n), z(n, n);
  for (int i = 0; i < n; ++i) z(i, i) = 1.0;
  const bool ok = schur(t, z);
  store(t, T);
  store(z, Z);
  return ok ? 1 : 0;
}

// min || rhs - H y ||, H m x n
void cd_lstsq(const double* H, int m, int n, const double* rhs, double* y) {
  CMat h = load(H, m, n);
  std::vector<Cx> r(m);
  std::memcpy(r.data(), rhs, sizeof(double) * 2 * m);
  const std::vector<Cx> out = lstsq(h, r);
  std::memcpy(y, out.data(), sizeof(double) * 2 * n);
}

// the deflated restart's algebra; Pk1 has room for (n+1) x (k+1), Hnew for
// (k+1) x k, c_r for k+1; returns the status (0 ok)
int cd_deflate(const double* H, int n, const double* res_vec, int k, double* Pk1, double* Hnew, double* c_r,
               int* k_eff) {
  CMat h = load(H, n + 1, n), p, hn;
  std::vector<Cx> rv(n + 1), cr;
  std::memcpy(rv.data(), res_vec, sizeof(double) * 2 * (n + 1));
  const int s = deflate_complex(h, rv, k, p, hn, cr);
  if (s) return s;
  *k_eff = hn.c;
  store(p, Pk1);
  store(hn, Hnew);
  std::memcpy(c_r, cr.data(), sizeof(double) * 2 * cr.size());
  return 0;
}

// Ritz (harmonic: harmonic Ritz) values of H ((n+1) x n); returns the count
int cd_ritz(const double* H, int n, int harmonic, double* ev) {
  CMat h = load(H, n + 1, n);
  std::vector<Cx> e;
  if (!ritz_values(h, harmonic != 0, e)) return -1;
  std::memcpy(ev, e.data(), sizeof(double) * 2 * e.size());
  return (int)e.size();
}

}  // extern "C"
