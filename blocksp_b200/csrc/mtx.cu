// mtx.cu — MatrixMarket (.mtx) coordinate files to block CSR and solArray order.
//
// Reference: blocksp_tests.hpp:582-699 (GotoLine, mtxMatrix_to_BlockSp,
// mtxArray_to_solArray).  Same file conventions:
//   * reading starts at line max(start_line, 1) (1-based; the line of the
//     size header "M N nnz" for a matrix, "M 1" for a vector);
//   * matrix entries "i j value", 1-based unless base_zero; a symmetric file
//     holds one triangle and (j, i) is filled with the same value;
//   * entry (i, j) lands in block (i / bs, j / bs) at (i % bs, j % bs); blocks
//     are created in order of first appearance and a repeated entry
//     overwrites, as util::setFromGlobal on a BlockSp does;
//   * a vector of M = n * B * D values fills a solArray<T, B, D> in its own
//     (element, dim, b) order.
// Two departures, both fixes: the reference's vector reader computes the
// in-block index as i % B instead of i % (B * D) (blocksp_tests.hpp:679), so
// for D > 1 every value lands in dim 0; here value i goes to flat position i.
// And the reference ignores base_zero (it always subtracts 1); here it is
// honoured.  Host code only: the result is handed to bsp_matrix_create.
#include <cstdio>
#include <fstream>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>
#include "internal.hpp"

namespace {

using bsp::record_error;

// Positions the stream at 1-based line `line` (0 and 1 both mean the first).
bool goto_line(std::ifstream& f, int line) {
  for (int i = 1; i < line; ++i) {
    std::string skip;
    if (!std::getline(f, skip)) return false;
  }
  return true;
}

}  // namespace

extern "C" {

int bsp_mtx_read_matrix(const char* path, int bs, int start_line, int symmetric, int base_zero, int* n_rows,
                        int* n_cols, int64_t* nnzb, int* row_ptr, int* col_idx, double* vals) {
  if (!path || bs < 1 || !n_rows || !n_cols || !nnzb) return BSP_INVALID;
  std::ifstream f(path);
  if (!f) {
    record_error(std::string("mtx: cannot open ") + path);
    return BSP_INVALID;
  }
  if (!goto_line(f, start_line)) {
    record_error("mtx: file shorter than start_line");
    return BSP_INVALID;
  }
  std::string line;
  long long M = 0, N = 0, nnz = 0;
  if (!std::getline(f, line) || std::sscanf(line.c_str(), "%lld %lld %lld", &M, &N, &nnz) != 3) {
    record_error("mtx: bad size line '" + line + "'");
    return BSP_INVALID;
  }
  if (M <= 0 || N <= 0 || nnz < 0 || M % bs || N % bs) {
    record_error("mtx: the block size must divide both matrix dimensions");
    return BSP_INVALID;
  }
  const int lm = (int)(M / bs), ln = (int)(N / bs);
  const int b2 = bs * bs;
  // blocks of each block row in order of first appearance
  std::vector<std::vector<int>> cols(lm);
  std::vector<std::unordered_map<int, int64_t>> where(lm);
  std::vector<int64_t> blk_row;          // block -> its block row
  std::vector<double> v;                 // block values, in creation order
  auto set = [&](long long i, long long j, double val) -> bool {
    if (i < 0 || j < 0 || i >= M || j >= N) return false;
    const int bi = (int)(i / bs), bj = (int)(j / bs);
    auto it = where[bi].find(bj);
    int64_t b;
    if (it == where[bi].end()) {
      b = (int64_t)blk_row.size();
      where[bi].emplace(bj, b);
      cols[bi].push_back(bj);
      blk_row.push_back(bi);
      v.resize(v.size() + b2, 0.0);
    } else {
      b = it->second;
    }
    v[b * b2 + (i % bs) * bs + (j % bs)] = val;
    return true;
  };
  const long long off = base_zero ? 0 : 1;
  for (long long k = 0; k < nnz; ++k) {
    long long i = 0, j = 0;
    double val = 0.0;
    if (!std::getline(f, line) || std::sscanf(line.c_str(), "%lld %lld %lf", &i, &j, &val) != 3) {
      record_error("mtx: entry " + std::to_string(k) + " unreadable");
      return BSP_INVALID;
    }
    i -= off;
    j -= off;
    if (!set(i, j, val) || (symmetric && i != j && !set(j, i, val))) {
      record_error("mtx: entry " + std::to_string(k) + " out of range");
      return BSP_INVALID;
    }
  }
  *n_rows = lm;
  *n_cols = ln;
  *nnzb = (int64_t)blk_row.size();
  if (!row_ptr) return BSP_OK;  // size query
  if (!col_idx || !vals) return BSP_INVALID;
  int64_t t = 0;
  row_ptr[0] = 0;
  for (int r = 0; r < lm; ++r) {
    for (int c : cols[r]) {
      const int64_t b = where[r].at(c);
      col_idx[t] = c;
      std::copy(v.begin() + b * b2, v.begin() + (b + 1) * b2, vals + t * b2);
      ++t;
    }
    row_ptr[r + 1] = (int)t;
  }
  return BSP_OK;
}

int bsp_mtx_read_vector(const char* path, int start_line, int B, int D, int64_t* n_values, double* out) {
  if (!path || B < 1 || D < 1 || !n_values) return BSP_INVALID;
  std::ifstream f(path);
  if (!f) {
    record_error(std::string("mtx: cannot open ") + path);
    return BSP_INVALID;
  }
  if (!goto_line(f, start_line)) {
    record_error("mtx: file shorter than start_line");
    return BSP_INVALID;
  }
  std::string line;
  long long M = 0, N = 0;
  if (!std::getline(f, line) || std::sscanf(line.c_str(), "%lld %lld", &M, &N) != 2 || N != 1 || M < 0 ||
      M % ((long long)B * D)) {
    record_error("mtx: a vector file of M x 1 values with B * D dividing M is required");
    return BSP_INVALID;
  }
  *n_values = M;
  if (!out) return BSP_OK;  // size query
  for (long long i = 0; i < M; ++i) {
    if (!std::getline(f, line) || std::sscanf(line.c_str(), "%lf", out + i) != 1) {
      record_error("mtx: value " + std::to_string(i) + " unreadable");
      return BSP_INVALID;
    }
  }
  return BSP_OK;
}

}  // extern "C"
