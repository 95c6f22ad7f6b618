// dropin_test.cpp — the same program solves one system with the reference
// BlockSp v1.0 (CPU, its own headers) and with include/blocksp_b200.hpp (GPU),
// through the same containers and the same call shapes, and prints how far
// apart the answers are.  Built by oracle/Makefile (it needs the reference
// headers); run by tests/test_dropin_gpu.py.
//
// usage: dropin_test <system.bsps> B D
//        dropin_test <system.bspc> B 1     (T = std::complex<double>)
// output: "CHECK <solver> <rel max-norm x difference> <ref iters> <gpu iters>"
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "blocksp_include.hpp"
#include "blocksp_b200.hpp"

namespace {

struct Sys {
  int n = 0, bs = 0, nrhs = 1;
  long long nnzb = 0;
  std::vector<int> row_ptr, col_idx;
  std::vector<double> vals, b;
};

Sys read_sys(const char* path) {
  Sys s;
  std::ifstream f(path, std::ios::binary);
  char magic[4];
  int ver = 0;
  f.read(magic, 4);
  f.read((char*)&ver, 4);
  f.read((char*)&s.n, 4);
  f.read((char*)&s.bs, 4);
  f.read((char*)&s.nnzb, 8);
  f.read((char*)&s.nrhs, 4);
  s.row_ptr.resize(s.n + 1);
  s.col_idx.resize(s.nnzb);
  s.vals.resize((size_t)s.nnzb * s.bs * s.bs);
  s.b.resize((size_t)s.n * s.bs * s.nrhs);
  f.read((char*)s.row_ptr.data(), 4 * (s.n + 1));
  f.read((char*)s.col_idx.data(), 4 * s.nnzb);
  f.read((char*)s.vals.data(), 8 * s.vals.size());
  f.read((char*)s.b.data(), 8 * s.b.size());
  return s;
}

template <int B, int D>
double rel_diff(const BlockSp::solArray<double, B, D>& x, const BlockSp::solArray<double, B, D>& y) {
  double num = 0.0, den = 0.0;
  for (int i = 0; i < x.len(); ++i)
    for (int d = 0; d < D; ++d)
      for (int b = 0; b < B; ++b) {
        num = std::fmax(num, std::fabs(x(i, d)(b) - y(i, d)(b)));
        den = std::fmax(den, std::fabs(y(i, d)(b)));
      }
  return num / den;
}

// iteration count from the reference's "pCG iters N" / "pGMRES iters N" line
int iters_of(const std::string& out) {
  const auto p = out.rfind("iters ");
  return p == std::string::npos ? -1 : std::stoi(out.substr(p + 6));
}

template <class F> std::string capture(F&& f) {
  std::stringstream buf;
  auto* old = std::cout.rdbuf(buf.rdbuf());
  f();
  std::cout.rdbuf(old);
  return buf.str();
}

template <int B, int D>
int run(const Sys& s) {
  constexpr int N = B * D;
  BlockSp::BlockSp<double, N> A(s.n);
  for (int i = 0; i < s.n; ++i)
    for (int t = s.row_ptr[i]; t < s.row_ptr[i + 1]; ++t) {
      blitz::TinyMatrix<double, N, N> m;
      std::memcpy(m.data(), &s.vals[(size_t)t * N * N], sizeof(double) * N * N);
      A(i, s.col_idx[t]) = m;
    }
  BlockSp::solArray<double, B, D> b(s.n);
  for (int i = 0; i < s.n; ++i)
    for (int d = 0; d < D; ++d)
      for (int k = 0; k < B; ++k) b(i, d)(k) = s.b[(size_t)i * N + d * B + k];

  // b = A x for a known x, both ways
  {
    auto y_ref = BlockSp::bsmv(A, b);
    auto y_gpu = blocksp_b200::bsmv<double, B, D>(A, b);
    std::printf("CHECK bsmv %.3e 0 0\n", rel_diff(y_gpu, y_ref));
  }
  // block algebra: identical structure (block order per row) and values
  {
    auto same = [](const BlockSp::BlockSp<double, N>& X, const BlockSp::BlockSp<double, N>& Y) {
      double num = 0.0, den = 0.0;
      bool structure = X.m() == Y.m();
      for (int i = 0; structure && i < X.m(); ++i) {
        const auto& cx = X.get_colIndex(i);
        const auto& cy = Y.get_colIndex(i);
        structure = cx.size() == cy.size() && std::equal(cx.begin(), cx.end(), cy.begin());
        for (size_t t = 0; structure && t < cx.size(); ++t)
          for (int e = 0; e < N * N; ++e) {
            num = std::fmax(num, std::fabs(X.get_data(i)[t].data()[e] - Y.get_data(i)[t].data()[e]));
            den = std::fmax(den, std::fabs(Y.get_data(i)[t].data()[e]));
          }
      }
      return structure ? num / den : 1.0;
    };
    std::printf("CHECK bsmm %.3e 0 0\n", same(blocksp_b200::bsmm<double, N>(A, A), BlockSp::bsmm<double, N>(A, A)));
    std::printf("CHECK bsmm_t %.3e 0 0\n",
                same(blocksp_b200::bsmm<double, N>(A, A, true), BlockSp::bsmm<double, N>(A, A, true)));
    std::printf("CHECK bs_tr %.3e 0 0\n", same(blocksp_b200::bs_tr<double, N>(A), BlockSp::bs_tr<double, N>(A)));
    std::printf("CHECK bs_id %.3e 0 0\n",
                same(blocksp_b200::bs_id<double, N>(s.n), BlockSp::bs_id<double, N>(s.n)));
    // Ritz values of A from 12 Arnoldi steps: largest magnitude and the real range
    BlockSp::preConditioners::NoPre<double, N, 1>* none = nullptr;
    auto er = BlockSp::arnoldi_eigenvalues<double, N>(A, 12, none);
    auto eg = blocksp_b200::arnoldi_eigenvalues<double, N>(A, 12);
    const double d = std::fmax(std::fabs(eg.max_mag() - er.max_mag()) / er.max_mag(),
                               std::fmax(std::fabs(eg.max_real() - er.max_real()) / er.max_mag(),
                                         std::fabs(eg.min_real() - er.min_real()) / er.max_mag()));
    std::printf("CHECK arnoldi_eig %.3e %d %d\n", d, (int)er.WR.size(), (int)eg.WR.size());
  }
  const double tol = 1e-10;
  {
    BlockSp::solArray<double, B, D> xr, xg;
    const std::string ro = capture([&] { xr = BlockSp::ILU0_pGMRES<double, B, D>(A, tol, 5000, 30, 10, true).solve(A, b); });
    const std::string go = capture([&] {
      xg = blocksp_b200::ILU0_pGMRES<double, B, D>(A, tol, 5000, 30, 10, true).solve(A, b);
    });
    std::printf("CHECK ilu0_pgmres_dr %.3e %d %d\n", rel_diff(xg, xr), iters_of(ro), iters_of(go));
  }
  {
    BlockSp::solArray<double, B, D> xr, xg;
    const std::string ro = capture([&] { xr = BlockSp::SOR_pGMRES<double, B, D>(A, 1.6, 3, 0, tol, 5000, -1, -1, true).solve(A, b); });
    const std::string go = capture([&] {
      xg = blocksp_b200::SOR_pGMRES<double, B, D>(A, 1.6, 3, 0, tol, 5000, -1, -1, true).solve(A, b);
    });
    std::printf("CHECK sor_pgmres %.3e %d %d\n", rel_diff(xg, xr), iters_of(ro), iters_of(go));
  }
  if (s.nrhs >= 1 && std::getenv("DROPIN_SPD")) {
    BlockSp::solArray<double, B, D> xr, xg;
    const std::string ro = capture([&] { xr = BlockSp::IChol0_pCG<double, B, D>(A, tol, 5000, true).solve(A, b); });
    const std::string go = capture([&] { xg = blocksp_b200::IChol0_pCG<double, B, D>(A, tol, 5000, true).solve(A, b); });
    std::printf("CHECK ichol0_pcg %.3e %d %d\n", rel_diff(xg, xr), iters_of(ro), iters_of(go));
    const std::string ro2 = capture([&] { xr = BlockSp::SOR_pCG<double, B, D>(A, 1.6, 3, tol, 5000, true).solve(A, b); });
    const std::string go2 = capture([&] { xg = blocksp_b200::SOR_pCG<double, B, D>(A, 1.6, 3, tol, 5000, true).solve(A, b); });
    std::printf("CHECK sor_pcg %.3e %d %d\n", rel_diff(xg, xr), iters_of(ro2), iters_of(go2));
  }
  return 0;
}

// ---- T = std::complex<double>: a "BSPC" file (values as (re, im) doubles)
struct CSys {
  int n = 0, bs = 0;
  long long nnzb = 0;
  std::vector<int> row_ptr, col_idx;
  std::vector<std::complex<double>> vals, b;
};

CSys read_csys(const char* path) {
  CSys s;
  std::ifstream f(path, std::ios::binary);
  char magic[4];
  int ver = 0, nrhs = 1;
  f.read(magic, 4);
  f.read((char*)&ver, 4);
  f.read((char*)&s.n, 4);
  f.read((char*)&s.bs, 4);
  f.read((char*)&s.nnzb, 8);
  f.read((char*)&nrhs, 4);
  s.row_ptr.resize(s.n + 1);
  s.col_idx.resize(s.nnzb);
  s.vals.resize((size_t)s.nnzb * s.bs * s.bs);
  s.b.resize((size_t)s.n * s.bs);
  f.read((char*)s.row_ptr.data(), 4 * (s.n + 1));
  f.read((char*)s.col_idx.data(), 4 * s.nnzb);
  f.read((char*)s.vals.data(), 16 * s.vals.size());
  f.read((char*)s.b.data(), 16 * s.b.size());
  return s;
}

template <int B>
double crel_diff(const BlockSp::solArray<std::complex<double>, B, 1>& x,
                 const BlockSp::solArray<std::complex<double>, B, 1>& y) {
  double num = 0.0, den = 0.0;
  for (int i = 0; i < x.len(); ++i)
    for (int b = 0; b < B; ++b) {
      num = std::fmax(num, std::abs(x(i, 0)(b) - y(i, 0)(b)));
      den = std::fmax(den, std::abs(y(i, 0)(b)));
    }
  return num / den;
}

template <int B>
int run_complex(const CSys& s) {
  using C = std::complex<double>;
  BlockSp::BlockSp<C, B> A(s.n);
  for (int i = 0; i < s.n; ++i)
    for (int t = s.row_ptr[i]; t < s.row_ptr[i + 1]; ++t) {
      blitz::TinyMatrix<C, B, B> m;
      for (int e = 0; e < B * B; ++e) m.data()[e] = s.vals[(size_t)t * B * B + e];
      A(i, s.col_idx[t]) = m;
    }
  BlockSp::solArray<C, B, 1> b(s.n);
  for (int i = 0; i < s.n; ++i)
    for (int k = 0; k < B; ++k) b(i, 0)(k) = s.b[(size_t)i * B + k];
  {
    auto y_ref = BlockSp::bsmv(A, b);
    auto y_gpu = blocksp_b200::bsmv<C, B, 1>(A, b);
    std::printf("CHECK c_bsmv %.3e 0 0\n", crel_diff(y_gpu, y_ref));
  }
  const double tol = 1e-10;
  {
    BlockSp::solArray<C, B, 1> xr, xg;
    const std::string ro = capture([&] { xr = BlockSp::ILU0_pGMRES<C, B, 1>(A, tol, 5000, 30, 10, true).solve(A, b); });
    const std::string go = capture([&] {
      xg = blocksp_b200::ILU0_pGMRES<C, B, 1>(A, tol, 5000, 30, 10, true).solve(A, b);
    });
    std::printf("CHECK c_ilu0_pgmres_dr %.3e %d %d\n", crel_diff(xg, xr), iters_of(ro), iters_of(go));
  }
  {
    BlockSp::solArray<C, B, 1> xr, xg;
    const std::string ro = capture([&] { xr = BlockSp::SOR_pGMRES<C, B, 1>(A, 1.2, 2, 0, tol, 5000, -1, -1, true).solve(A, b); });
    const std::string go = capture([&] {
      xg = blocksp_b200::SOR_pGMRES<C, B, 1>(A, 1.2, 2, 0, tol, 5000, -1, -1, true).solve(A, b);
    });
    std::printf("CHECK c_sor_pgmres %.3e %d %d\n", crel_diff(xg, xr), iters_of(ro), iters_of(go));
  }
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 4) {
    std::fprintf(stderr, "usage: dropin_test <system.bsps> B D\n");
    return 2;
  }
  const int B = std::atoi(argv[2]), D = std::atoi(argv[3]);
  {
    char magic[4] = {0, 0, 0, 0};
    std::ifstream f(argv[1], std::ios::binary);
    f.read(magic, 4);
    if (std::memcmp(magic, "BSPC", 4) == 0) {
      const CSys cs = read_csys(argv[1]);
      try {
        if (B == 2 && D == 1) return run_complex<2>(cs);
        if (B == 4 && D == 1) return run_complex<4>(cs);
      } catch (const blocksp_b200::error& e) {
        std::printf("ERROR %d %s\n", e.status, e.what());
        return 1;
      }
      std::fprintf(stderr, "unsupported complex B\n");
      return 2;
    }
  }
  const Sys s = read_sys(argv[1]);
  try {
    if (B == 2 && D == 2) return run<2, 2>(s);
    if (B == 4 && D == 2) return run<4, 2>(s);
    if (B == 4 && D == 1) return run<4, 1>(s);
  } catch (const blocksp_b200::error& e) {
    std::printf("ERROR %d %s\n", e.status, e.what());
    return 1;
  }
  std::fprintf(stderr, "unsupported (B, D)\n");
  return 2;
}
