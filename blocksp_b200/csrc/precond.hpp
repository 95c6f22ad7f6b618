// precond.hpp — host-side state of a block preconditioner (shared by the
// single-system, batched and learned solvers).
#pragma once
#include "internal.hpp"
#include "sweep_stream.hpp"

namespace bsp {
// Elimination plan of a block ILU0 / IChol0 factorisation (pattern only).
// For every strictly-lower factor entry e (block (k, i)), the updates it makes
// to later blocks of its own row k, in the reference's order:
// pairs[pp[e] .. pp[e+1]) = {target factor entry, source}, where source >= 0
// is a factor entry of another row (U_ij for ILU0: A_kj -= L_ki U_ij; L_ji
// for IChol0: A_kj -= L_ki L_ji^T) and source < 0 names the entry -1 - source
// of row k itself (IChol0's diagonal update A_kk -= L_ki L_ki^T).
struct FactorPlan {
  DevBuf<int> pp;        // f_nnzb + 1
  DevBuf<int2> pairs;
  int max_row = 0;       // blocks of the longest factor row
  int max_deps = 0;      // largest per-entry dependency count (inverse diagonal + sources)
};
}  // namespace bsp

struct bsp_precond_s {
  bsp_handle_t h = nullptr;
  int device = 0;
  bsp_matrix_t A = nullptr;
  int kind = 0, n = 0, bs = 0, precision = 0;
  double w = 1.6;
  // learned factors: off-diagonal factor blocks scaled by (1 + relax) before the
  // network's correction is added
  double relax = 0.0;
  int nu = 3, type = 0;
  // factor storage (ILU0: every block of A; IChol0: A.lowTri()), columns sorted
  bsp::DevBuf<int> f_ptr, f_col, f_diag;
  bsp::DevBuf<double> f_vals;
  bsp::DevBuf<float> f_vals32;
  bsp::DevBuf<__nv_bfloat16> f_vals16;
  std::vector<int64_t> h_perm;  // factor entry -> block index in A
  bsp::DevBuf<int64_t> d_perm;
  int64_t f_nnzb = 0;
  // IChol0 backward sweep: transposed strictly-lower structure of L
  bsp::DevBuf<int> t_ptr, t_row;
  bsp::DevBuf<int64_t> t_blk;
  // SOR / Diag on A's own structure
  bsp::DevBuf<int> a_diag;
  // inverted diagonal blocks (U_ii^-1, L_ii^-1 or A_ii^-1)
  bsp::DevBuf<double> dinv;
  bsp::DevBuf<float> dinv32;
  bsp::DevBuf<__nv_bfloat16> dinv16;
  // level orders
  bsp::DevBuf<int> order_lo, order_up;
  int n_lev_lo = 0, n_lev_up = 0;
  // chains of consecutive dependent rows, in chain-level order (sweep tasks)
  bsp::DevBuf<int> task_lo_row, task_lo_len, task_up_row, task_up_len;
  int n_task_lo = 0, n_task_up = 0;
  // sync-free state
  bsp::DevBuf<int> flags;
  bsp::DevBuf<unsigned> ticket;
  // transposed solves M^-T = L^-T U^-T of an LU-type factor (built on demand):
  // tu lists, per column j, the strictly-upper blocks (i, j); tl, per column i,
  // the strictly-lower blocks (j, i); each with its own chain tasks
  bool has_trans = false;
  bsp::DevBuf<int> tu_ptr, tu_row, tl_ptr, tl_row, order_tu, order_tl, task_tu_row, task_tu_len, task_tl_row,
      task_tl_len;
  bsp::DevBuf<int64_t> tu_blk, tl_blk;
  int n_task_tu = 0, n_task_tl = 0;
  // apply scratch: sweep outputs (pre-filled with the sentinel), SOR ping-pong
  // iterates and the copy of an in-place right-hand side
  bsp::DevBuf<double> s64[3];
  bsp::DevBuf<float> s32[3];
  // streamed sweeps (ILU0 / IChol0 and the learned factors, FP64 vectors):
  // the layout, shared with the matrix's symbolic cache, and its values per
  // precision (index BSP_PREC_*), gathered from f_vals / dinv on first use
  // after every change of the factors
  std::shared_ptr<bsp::StreamSym> ss_lo, ss_up;
  bsp::StreamVals sv_lo[3], sv_up[3];
  // elimination plan of the factorisation (shared with the matrix's cache)
  std::shared_ptr<bsp::FactorPlan> plan;
};

namespace bsp {
int grid_for(const bsp_handle_s* h, int64_t n, int threads);
int precond_build(bsp_precond_s* pc);
int precond_apply(bsp_precond_s* pc, int precision, const void* r, void* z);
int precond_check_status(bsp_precond_s* pc);
// out = M^-T g for an ILU0 / learned-LU preconditioner (FP64); w receives U^-T g.
int precond_apply_transposed(bsp_precond_s* pc, const double* g, double* w, double* out);
// learned LU: structure only (no factorisation), then
// f = ilu's factors (off-diagonal blocks scaled by 1 + work->relax) + dF
// (A's block order) with dinv recomputed
int precond_learned_init(bsp_precond_s* pc);
int precond_learned_refresh(bsp_precond_s* work, const bsp_precond_s* ilu, const double* dF);
}  // namespace bsp
