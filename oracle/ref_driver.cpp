// oracle/ref_driver.cpp — runs the reference BlockSp v1.0 solve path on a system file.
//
// TEST INFRASTRUCTURE ONLY.  Compiled by oracle/Makefile against the
// reference's own headers (unmodified for the timed build; with the
// reference's commented-out residual prints enabled for the history build)
// and the shims in oracle/shim.  Used as the checker that pins the numpy
// oracle, to make golden fixtures, and as the timed CPU baseline.
//
// usage: ref_solve <system.bsps> --B b --D d --solver NAME [options]
//   solvers: bsmv | bsmv_multi | ilu0_pgmres | sor_pgmres | nopre_pgmres |
//            ichol0_pcg | sor_pcg | diag_pcg | nopre_pcg |
//            ilu0_apply | ichol0_apply | sor_apply | diag_apply |
//            bsmm (--atran 0/1) | bs_tr | pseudo_heat (--delta d): result matrix to --x |
//            arnoldi_eig | arnoldi_eig_ilu0 (--maxit = iters, --k 1: harmonic Ritz)
//   options: --tol t --maxit m --restart r --k k --w w --nu nu --sortype t
//            --reps n (bsmv) --x out.vec --time --print-iters
//   LDG known answer: ref_solve --ldg <dir with LDG_2D_vecLap*.mtx> --B b
// Output lines: "RES0 ..", "RES it res" (history build), "ITERS n",
// "TIME setup_s v", "TIME solve_s v", "ERRINF v".
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <string>
#include <vector>
#include "blocksp_include.hpp"
#include "blocksp_tests.hpp"

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
  if (!f) {
    std::fprintf(stderr, "cannot open %s\n", path);
    std::exit(2);
  }
  char magic[4];
  f.read(magic, 4);
  int ver = 0;
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

void write_vec(const std::string& path, const double* v, long long m) {
  std::ofstream f(path, std::ios::binary);
  f.write((const char*)&m, 8);
  f.write((const char*)v, 8 * m);
}

// A BlockSp (and right-hand side b) in the exchange format read_sys reads.
template <int N>
void write_blocksp(const std::string& path, const BlockSp::BlockSp<double, N>& A, const std::vector<double>& b) {
  std::vector<int> rp{0}, ci;
  std::vector<double> v;
  for (int i = 0; i < A.m(); ++i) {
    const auto& blocks = A.get_data(i);
    const auto& cols = A.get_colIndex(i);
    for (size_t t = 0; t < blocks.size(); ++t) {
      ci.push_back(cols[t]);
      v.insert(v.end(), blocks[t].data(), blocks[t].data() + N * N);
    }
    rp.push_back((int)ci.size());
  }
  std::ofstream f(path, std::ios::binary);
  const int ver = 1, n = A.m(), bs = N, nrhs = 1;
  const long long nnzb = (long long)ci.size();
  f.write("BSPS", 4);
  f.write((const char*)&ver, 4);
  f.write((const char*)&n, 4);
  f.write((const char*)&bs, 4);
  f.write((const char*)&nnzb, 8);
  f.write((const char*)&nrhs, 4);
  f.write((const char*)rp.data(), 4 * rp.size());
  f.write((const char*)ci.data(), 4 * ci.size());
  f.write((const char*)v.data(), 8 * v.size());
  std::vector<double> bb(b);
  bb.resize((size_t)n * N, 0.0);
  f.write((const char*)bb.data(), 8 * bb.size());
}

struct Opts {
  std::string solver = "ilu0_pgmres", xout, ldg;
  double tol = 1e-10, w = 1.6, delta = 2e-4;
  int atran = 0;
  int maxit = 5000, restart = -1, k = -1, nu = 3, sortype = 0, reps = 1, B = 0, D = 1;
  bool time = false, print_iters = false;
};

double now() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// BSR arrays -> the reference container, blocks inserted in stored order.
template <int N>
BlockSp::BlockSp<double, N> to_blocksp(const Sys& s) {
  BlockSp::BlockSp<double, N> A(s.n);
  for (int i = 0; i < s.n; ++i)
    for (int t = s.row_ptr[i]; t < s.row_ptr[i + 1]; ++t) {
      blitz::TinyMatrix<double, N, N> m;
      std::memcpy(m.data(), &s.vals[(size_t)t * N * N], sizeof(double) * N * N);
      A(i, s.col_idx[t]) = m;
    }
  A.shrink_to_fit();
  return A;
}

template <int B, int D>
BlockSp::solArray<double, B, D> to_sol(const double* v, int n) {
  BlockSp::solArray<double, B, D> x(n);
  for (int i = 0; i < n; ++i)
    for (int d = 0; d < D; ++d)
      for (int b = 0; b < B; ++b) x(i, d)(b) = v[(size_t)i * B * D + d * B + b];
  return x;
}

template <int B, int D>
void from_sol(const BlockSp::solArray<double, B, D>& x, std::vector<double>& v) {
  v.resize((size_t)x.len() * B * D);
  for (int i = 0; i < x.len(); ++i)
    for (int d = 0; d < D; ++d)
      for (int b = 0; b < B; ++b) v[(size_t)i * B * D + d * B + b] = x(i, d)(b);
}

template <int B, int D, class Pre>
void print_res0(const BlockSp::solArray<double, B, D>& b, const Pre& pre) {
  auto r0{b};
  pre(r0);
  std::cout << "RES0 " << BlockSp::twoNorm<double, B, D>(r0, r0) << "\n";
}

template <int B, int D>
int run(const Sys& s, const Opts& o) {
  constexpr int N = B * D;
  using namespace BlockSp;
  std::vector<double> xv;
  if (o.solver == "bsmv_multi") {  // BlockSp<T,B> x solArray<T,B,D>, dims independent
    auto A = to_blocksp<B>(s);
    auto x = to_sol<B, D>(s.b.data(), s.n);
    solArray<double, B, D> y;
    const double t0 = now();
    for (int r = 0; r < o.reps; ++r) y = bsmv<double, B, D>(A, x);
    const double t1 = now();
    from_sol(y, xv);
    if (o.time) std::cout << "TIME bsmv_s " << (t1 - t0) / o.reps << "\n";
  } else {
    if (s.bs != N) {
      std::fprintf(stderr, "system block size %d != B*D = %d\n", s.bs, N);
      return 2;
    }
    auto A = to_blocksp<N>(s);
    auto b = to_sol<B, D>(s.b.data(), s.n);
    solArray<double, B, D> x;
    double t0 = now(), t1 = t0, t2 = t0;
    const std::string& sv = o.solver;
    if (sv == "arnoldi_eig" || sv == "arnoldi_eig_ilu0") {
      // arnoldi_eigenvalues (blocksp_solvers.hpp:306-334): one EIG line per value
      auto print = [](const dense::Eigenvalues_Arr<double>& e) {
        for (int i = 0; i < e.N; ++i) std::cout << "EIG " << e.WR(i) << " " << e.WI(i) << "\n";
      };
      if (sv == "arnoldi_eig") {
        const preConditioners::NoPre<double, N, 1>* none = nullptr;
        print(arnoldi_eigenvalues<double, N>(A, o.maxit, none, false, false, o.k > 0));
      } else {
        preConditioners::ILU0<double, N, 1> pre(A);
        print(arnoldi_eigenvalues<double, N>(A, o.maxit, &pre, false, false, o.k > 0));
      }
      return 0;
    }
    if (sv == "bsmm" || sv == "bs_tr" || sv == "pseudo_heat") {
      // block algebra: the result matrix is written to --x in the exchange format
      if (sv == "bsmm") write_blocksp<N>(o.xout, bsmm<double, N>(A, A, o.atran != 0), s.b);
      else if (sv == "bs_tr") write_blocksp<N>(o.xout, bs_tr<double, N>(A), s.b);
      else  // block_pseudo_heat's operator (blocksp_tests.hpp:282-285)
        write_blocksp<N>(o.xout, bs_id<double, N>(s.n) - o.delta * bsmm(A, A, true), s.b);
      return 0;
    }
    if (sv == "bsmv") {
      t1 = now();
      for (int r = 0; r < o.reps; ++r) {
        solArray<double, B, D> y(s.n);
        bsmv<double, B, D>(y, A, b);  // the accumulating void overload
        if (r + 1 == o.reps) x = y;
      }
      t2 = now();
      if (o.time) std::cout << "TIME bsmv_s " << (t2 - t1) / o.reps << "\n";
    } else if (sv == "ilu0_pgmres") {
      ILU0_pGMRES<double, B, D> solver(A, o.tol, o.maxit, o.restart, o.k, o.print_iters);
      t1 = now();
      print_res0(b, solver.access_ILU0_pre());
      x = solver.solve(A, b);
      t2 = now();
    } else if (sv == "sor_pgmres") {
      SOR_pGMRES<double, B, D> solver(A, o.w, o.nu, o.sortype, o.tol, o.maxit, o.restart, o.k,
                                      o.print_iters);
      t1 = now();
      print_res0(b, solver.access_SOR_pre());
      x = solver.solve(A, b);
      t2 = now();
    } else if (sv == "nopre_pgmres") {
      preConditioners::NoPre<double, B, D> np;
      t1 = now();
      print_res0(b, np);
      x = pGMRES<double, B, D>(A, b, o.tol, np, o.maxit, o.restart, o.k, o.print_iters);
      t2 = now();
    } else if (sv == "ichol0_pcg") {
      IChol0_pCG<double, B, D> solver(A, o.tol, o.maxit, o.print_iters);
      t1 = now();
      x = solver.solve(A, b);
      t2 = now();
    } else if (sv == "sor_pcg") {
      SOR_pCG<double, B, D> solver(A, o.w, o.nu, o.tol, o.maxit, o.print_iters);
      t1 = now();
      x = solver.solve(A, b);
      t2 = now();
    } else if (sv == "diag_pcg") {
      preConditioners::Diag<dense::CholeskyFactor<double, N>, double, B, D> pre(A);
      t1 = now();
      x = pCG<double, B, D>(A, b, o.tol, pre, o.maxit, o.print_iters);
      t2 = now();
    } else if (sv == "nopre_pcg") {
      preConditioners::NoPre<double, B, D> np;
      t1 = now();
      x = pCG<double, B, D>(A, b, o.tol, np, o.maxit, o.print_iters);
      t2 = now();
    } else if (sv == "ilu0_apply") {
      preConditioners::ILU0<double, B, D> pre(A);
      t1 = now();
      x = b;
      for (int r = 0; r < o.reps; ++r) {
        x = b;
        pre(x);
      }
      t2 = now();
    } else if (sv == "ichol0_apply") {
      preConditioners::IChol0<double, B, D> pre(A);
      t1 = now();
      for (int r = 0; r < o.reps; ++r) {
        x = b;
        pre(x);
      }
      t2 = now();
    } else if (sv == "sor_apply") {
      preConditioners::SOR<dense::LUFactor<double, N>, double, B, D> pre(A, o.w, o.nu, o.sortype);
      t1 = now();
      for (int r = 0; r < o.reps; ++r) {
        x = b;
        pre(x);
      }
      t2 = now();
    } else if (sv == "diag_apply") {
      preConditioners::Diag<dense::LUFactor<double, N>, double, B, D> pre(A);
      t1 = now();
      for (int r = 0; r < o.reps; ++r) {
        x = b;
        pre(x);
      }
      t2 = now();
    } else {
      std::fprintf(stderr, "unknown solver %s\n", sv.c_str());
      return 2;
    }
    if (o.time) {
      std::cout << "TIME setup_s " << (t1 - t0) << "\n";
      std::cout << "TIME solve_s " << (t2 - t1) / (sv.find("apply") != std::string::npos ? o.reps : 1) << "\n";
    }
    from_sol(x, xv);
  }
  if (!o.xout.empty()) write_vec(o.xout, xv.data(), (long long)xv.size());
  return 0;
}

// The reference's LDG known answer (blocksp_tests.hpp:304-342): infinity-norm
// error of the solution against the exact one, per solver, at tol 1e-8.
template <int B>
int run_ldg(const Opts& o) {
  using namespace BlockSp;
  const std::string d = o.ldg;
  auto A = tests::mtxMatrix_to_BlockSp<double, B>(d + "/LDG_2D_vecLap.mtx", 1, true);
  A.shrink_to_fit();
  auto xe = tests::mtxArray_to_solArray<double, B, 1>(d + "/LDG_2D_vecLap_sol.mtx", 1);
  auto b = tests::mtxArray_to_solArray<double, B, 1>(d + "/LDG_2D_vecLap_b.mtx", 1);
  auto report = [&](const char* name, const solArray<double, B, 1>& x) {
    std::cout << "ERRINF " << name << " " << infNorm<double, B, 1>(x - xe) << "\n";
  };
  report("ichol0_pcg", IChol0_pCG<double, B, 1>(A, 1e-8, 5000, true).solve(A, b));
  report("ilu0_pgmres", ILU0_pGMRES<double, B, 1>(A, 1e-8, 5000, -1, -1, true).solve(A, b));
  report("ilu0_pgmres_dr", ILU0_pGMRES<double, B, 1>(A, 1e-8, 5000, 30, 10, true).solve(A, b));
  report("sor_pcg", SOR_pCG<double, B, 1>(A, 1.6, 3, 1e-8, 5000, true).solve(A, b));
  if (!o.xout.empty()) {
    std::vector<double> xv;
    from_sol(IChol0_pCG<double, B, 1>(A, 1e-8, 5000).solve(A, b), xv);
    write_vec(o.xout, xv.data(), (long long)xv.size());
  }
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
    else if (a == "--D") o.D = std::stoi(next());
    else if (a == "--tol") o.tol = std::stod(next());
    else if (a == "--maxit") o.maxit = std::stoi(next());
    else if (a == "--restart") o.restart = std::stoi(next());
    else if (a == "--k") o.k = std::stoi(next());
    else if (a == "--w") o.w = std::stod(next());
    else if (a == "--nu") o.nu = std::stoi(next());
    else if (a == "--sortype") o.sortype = std::stoi(next());
    else if (a == "--reps") o.reps = std::stoi(next());
    else if (a == "--atran") o.atran = std::stoi(next());
    else if (a == "--delta") o.delta = std::stod(next());
    else if (a == "--x") o.xout = next();
    else if (a == "--ldg") o.ldg = next();
    else if (a == "--time") o.time = true;
    else if (a == "--print-iters") o.print_iters = true;
    else sys_path = argv[i];
  }
  if (!o.ldg.empty()) {
    switch (o.B) {
      case 1: return run_ldg<1>(o);
      case 2: return run_ldg<2>(o);
      case 4: return run_ldg<4>(o);
      case 8: return run_ldg<8>(o);
      default: std::fprintf(stderr, "LDG: B must be 1, 2, 4 or 8\n"); return 2;
    }
  }
  if (!sys_path) {
    std::fprintf(stderr, "usage: ref_solve <system.bsps> --B b --D d --solver name [...]\n");
    return 2;
  }
  const Sys s = read_sys(sys_path);
#define BSP_CASE(BB, DD) \
  if (o.B == BB && o.D == DD) return run<BB, DD>(s, o);
  BSP_CASE(1, 1) BSP_CASE(2, 1) BSP_CASE(3, 1) BSP_CASE(4, 1) BSP_CASE(8, 1) BSP_CASE(16, 1)
  BSP_CASE(1, 2) BSP_CASE(2, 2) BSP_CASE(4, 2) BSP_CASE(8, 2) BSP_CASE(16, 2)
#undef BSP_CASE
  std::fprintf(stderr, "unsupported (B, D) = (%d, %d)\n", o.B, o.D);
  return 2;
}
