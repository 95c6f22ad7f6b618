// oracle/ref_complex.cpp — runs the reference BlockSp v1.0 solve path with
// T = std::complex<double> on a complex system file.
//
// TEST INFRASTRUCTURE ONLY.  Compiled by oracle/Makefile against the
// history-enabled copy of the reference headers (the same copy ref_solve_hist
// uses) and the shims in oracle/shim.  Makes the complex golden fixtures.
//
// usage: ref_complex <system.bspc> --B b --solver NAME [options]
//   solvers: bsmv | ilu0_apply | sor_apply | diag_apply |
//            ilu0_pgmres | sor_pgmres | diag_pgmres | nopre_pgmres
//   options: --tol t --maxit m --restart r --k k --w w --nu nu --sortype t --x out.vec
// The system file is the real exchange format with magic "BSPC": every value
// (blocks, right-hand side) is a complex number stored as (re, im) doubles.
// Output lines: "RES0 ..", "RES it res" (history build), "pGMRES iters n",
// "TIME setup_s v" / "TIME solve_s v" (ilu0_pgmres); --x writes
// the result vector as interleaved (re, im) doubles.
#include <chrono>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <string>
#include <vector>
#include "blocksp_include.hpp"

namespace {

using C = std::complex<double>;

struct Sys {
  int n = 0, bs = 0, nrhs = 1;
  long long nnzb = 0;
  std::vector<int> row_ptr, col_idx;
  std::vector<C> vals, b;
};

Sys read_sys(const char* path) {
  Sys s;
  std::ifstream f(path, std::ios::binary);
  if (!f) {
    std::fprintf(stderr, "cannot open %s\n", path);
    std::exit(2);
  }
  char magic[4];
  f.read(magic, 4);
  if (std::memcmp(magic, "BSPC", 4) != 0) {
    std::fprintf(stderr, "%s is not a complex system file\n", path);
    std::exit(2);
  }
  int ver = 0;
  f.read((char*)&ver, 4);
  f.read((char*)&s.n, 4);
  f.read((char*)&s.bs, 4);
  f.read((char*)&s.nnzb, 8);
  f.read((char*)&s.nrhs, 4);
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

struct Opts {
  std::string solver = "ilu0_pgmres", xout;
  double tol = 1e-10, w = 1.6;
  int maxit = 5000, restart = -1, k = -1, nu = 3, sortype = 0, B = 0;
};

template <int N>
BlockSp::BlockSp<C, N> to_blocksp(const Sys& s) {
  BlockSp::BlockSp<C, N> A(s.n);
  for (int i = 0; i < s.n; ++i)
    for (int t = s.row_ptr[i]; t < s.row_ptr[i + 1]; ++t) {
      blitz::TinyMatrix<C, N, N> m;
      for (int e = 0; e < N * N; ++e) m.data()[e] = s.vals[(size_t)t * N * N + e];
      A(i, s.col_idx[t]) = m;
    }
  A.shrink_to_fit();
  return A;
}

template <int N>
BlockSp::solArray<C, N, 1> to_sol(const std::vector<C>& v, int n) {
  BlockSp::solArray<C, N, 1> x(n);
  for (int i = 0; i < n; ++i)
    for (int b = 0; b < N; ++b) x(i, 0)(b) = v[(size_t)i * N + b];
  return x;
}

template <int N>
void write_sol(const std::string& path, const BlockSp::solArray<C, N, 1>& x) {
  if (path.empty()) return;
  std::vector<C> v((size_t)x.len() * N);
  for (int i = 0; i < x.len(); ++i)
    for (int b = 0; b < N; ++b) v[(size_t)i * N + b] = x(i, 0)(b);
  std::ofstream f(path, std::ios::binary);
  const long long m = (long long)v.size() * 2;
  f.write((const char*)&m, 8);
  f.write((const char*)v.data(), 16 * v.size());
}

template <int N, class Pre>
void print_res0(const BlockSp::solArray<C, N, 1>& b, const Pre& pre) {
  auto r0{b};
  pre(r0);
  std::cout << "RES0 " << BlockSp::twoNorm<C, N, 1>(r0, r0) << "\n";
}

template <int N>
int run(const Sys& s, const Opts& o) {
  using namespace BlockSp;
  if (s.bs != N) {
    std::fprintf(stderr, "system block size %d != B = %d\n", s.bs, N);
    return 2;
  }
  auto A = to_blocksp<N>(s);
  auto b = to_sol<N>(s.b, s.n);
  solArray<C, N, 1> x;
  using LU = dense::LUFactor<C, N>;
  const std::string& sv = o.solver;
  if (sv == "bsmv") {
    x = bsmv<C, N, 1>(A, b);
  } else if (sv == "ilu0_apply") {
    preConditioners::ILU0<C, N, 1> pre(A);
    x = b;
    pre(x);
  } else if (sv == "sor_apply") {
    preConditioners::SOR<LU, C, N, 1> pre(A, o.w, o.nu, o.sortype);
    x = b;
    pre(x);
  } else if (sv == "diag_apply") {
    preConditioners::Diag<LU, C, N, 1> pre(A);
    x = b;
    pre(x);
  } else if (sv == "ilu0_pgmres") {
    auto now = [] { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); };
    const double t0 = now();
    ILU0_pGMRES<C, N, 1> solver(A, o.tol, o.maxit, o.restart, o.k, true);
    const double t1 = now();
    print_res0(b, solver.access_ILU0_pre());
    const double t2 = now();
    x = solver.solve(A, b);
    const double t3 = now();
    std::cout << "TIME setup_s " << (t1 - t0) << "\nTIME solve_s " << (t3 - t2) << "\n";
  } else if (sv == "sor_pgmres") {
    SOR_pGMRES<C, N, 1> solver(A, o.w, o.nu, o.sortype, o.tol, o.maxit, o.restart, o.k, true);
    print_res0(b, solver.access_SOR_pre());
    x = solver.solve(A, b);
  } else if (sv == "diag_pgmres") {
    preConditioners::Diag<LU, C, N, 1> pre(A);
    print_res0(b, pre);
    x = pGMRES<C, N, 1>(A, b, o.tol, pre, o.maxit, o.restart, o.k, true);
  } else if (sv == "nopre_pgmres") {
    preConditioners::NoPre<C, N, 1> np;
    print_res0(b, np);
    x = pGMRES<C, N, 1>(A, b, o.tol, np, o.maxit, o.restart, o.k, true);
  } else {
    std::fprintf(stderr, "unknown solver %s\n", sv.c_str());
    return 2;
  }
  write_sol<N>(o.xout, x);
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  std::cout << std::setprecision(17);
  Opts o;
  const char* sys_path = nullptr;
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i];
    auto next = [&]() -> std::string {
      if (i + 1 >= argc) {
        std::fprintf(stderr, "missing value for %s\n", a.c_str());
        std::exit(2);
      }
      return argv[++i];
    };
    if (a == "--solver") o.solver = next();
    else if (a == "--B") o.B = std::stoi(next());
    else if (a == "--tol") o.tol = std::stod(next());
    else if (a == "--maxit") o.maxit = std::stoi(next());
    else if (a == "--restart") o.restart = std::stoi(next());
    else if (a == "--k") o.k = std::stoi(next());
    else if (a == "--w") o.w = std::stod(next());
    else if (a == "--nu") o.nu = std::stoi(next());
    else if (a == "--sortype") o.sortype = std::stoi(next());
    else if (a == "--x") o.xout = next();
    else sys_path = argv[i];
  }
  if (!sys_path) {
    std::fprintf(stderr, "usage: ref_complex <system.bspc> --B b --solver name [...]\n");
    return 2;
  }
  const Sys s = read_sys(sys_path);
  switch (o.B) {
    case 1: return run<1>(s, o);
    case 2: return run<2>(s, o);
    case 4: return run<4>(s, o);
    case 8: return run<8>(s, o);
    default: std::fprintf(stderr, "B must be 1, 2, 4 or 8\n"); return 2;
  }
}
