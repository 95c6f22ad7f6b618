// sweep_stream.hpp — the streamed triangular sweep: host-side interface.
//
// A sweep of a block triangular factor (ILU0: unit-L forward, U backward with
// the inverted diagonal; IChol0: L forward with L_ii^-1, L^T backward with
// L_ii^-T) computes, in the reference's natural row order,
//     x_r = D_r (rhs_r - sum_e B_e x_{j_e})
// (blocksp_preconditioners.hpp:294-349 ILU0::invmul, :432-489 IChol0::invmul),
// with D_r the identity for the unit-L sweep.  The streamed form lays every
// block the sweep reads out once, in the order the device consumes it:
//   * rows are grouped into chains (runs of consecutive rows, each depending
//     on the one before; at most kStreamCmax rows), chains into super-tasks of
//     W chains (one CTA, one warp per chain).  When one chain stride d links
//     at least half of the chains (the neighbouring plane of a grid), a
//     super-task is a tile of wy consecutive chains by wz chains d apart, so
//     both directions across the chains are handed over inside the CTA;
//     otherwise it is W consecutive chains;
//   * super-tasks are sorted by dependency level (the ticket order);
//   * per row the entries are ordered external rows first, rows of the same
//     super-task next, the chain's previous row last, and each entry carries a
//     code: >= 0 an external row (published through global memory), -1 the
//     chain's previous row (registers), <= -2 a row of another chain of the
//     same CTA (shared memory);
//   * the blocks (transposed where the sweep reads B^T) and the D blocks are
//     stored contiguously in that order, in the precision of the solve; in a
//     sweep with D blocks every block is stored premultiplied by its row's D,
//     x_r = D_r rhs_r - sum_e (D_r B_e) x_{j_e}, so D_r rhs_r is formed before
//     the row's dependencies arrive and D leaves the dependency path (the same
//     operator; the rounding of the two products differs).
// What a row computes is unchanged; only when it runs and where its inputs
// come from differ from the reference's loop.
#pragma once
#include <memory>
#include <vector>
#include "internal.hpp"

namespace bsp {

constexpr int kStreamEmax = 3;   // entries of a row staged in shared memory
constexpr int kStreamCmax = 64;  // rows per chain (longer runs are split)

// Symbolic part of one streamed sweep (depends on the matrix pattern only).
struct StreamSym {
  int n = 0, n_super = 0, n_chains = 0, W = 0, dir = 1;
  int n_levels = 0, stride = 0;  // super-task levels; chain stride of the tiles (0: consecutive)
  int64_t n_ent = 0;
  bool trans_blocks = false, has_d = false, trans_d = false;
  DevBuf<int> super_beg;   // n_super + 1: chains of each super-task (ticket order, warp order)
  DevBuf<int4> chains;     // {row0, len, q0 (first stream row), e0 (first entry)}
  DevBuf<int4> rec;        // per stream row: {code0, code1, code2, n_entries}
  DevBuf<int> codes;       // per entry (rows with more than kStreamEmax entries)
  DevBuf<int64_t> src_blk; // per entry: block index in the factor's value array
  DevBuf<int> q_row;       // per stream row: its block row (D gather)
  DevBuf<int> ent_q;       // per entry: its stream row (D-premultiplied gather)
};

// The entries of a sweep in CSR form: row i reads rows col[t] through the
// factor blocks blk[t], t in [ptr[i], ptr[i+1]).
struct SweepEntries {
  std::vector<int> ptr, col;
  std::vector<int64_t> blk;
};

// The layout of a sweep on the host (the arrays StreamSym holds on the device).
struct StreamPlan {
  int n = 0, n_super = 0, n_chains = 0, W = 0, dir = 1, n_levels = 0, stride = 0;
  std::vector<int> super_beg, codes, q_row, ent_q;
  std::vector<int4> chains, rec;
  std::vector<int64_t> src_blk;
};
int stream_plan(int n, bool ascending, int warps, const SweepEntries& ent, StreamPlan& P);

// Builds the streamed layout of a sweep over n rows; ascending: forward
// sweep (dependencies j < i), else backward (j > i).
int stream_build(int n, bool ascending, int warps, const SweepEntries& ent, bool trans_blocks, bool has_d,
                 bool trans_d, StreamSym& S);

// Block size, precision and warp count the streamed kernel supports.
bool stream_supported(int bs);
int stream_warps(int bs);

// Per-precision values of one streamed sweep.
struct StreamVals {
  DevBuf<unsigned char> vals, dvals;  // blocks, D blocks (VT)
  bool valid = false;
};

// Bytes of the stream's blocks and D blocks in precision prec.
size_t stream_val_bytes(const StreamSym& S, int bs, int prec);
size_t stream_dval_bytes(const StreamSym& S, int bs, int prec);

// Gathers the stream's values (into buffers of at least the sizes above)
// from the factor (FP64, factor entry order) and
// the D blocks from dinv (FP64, row order), converted to the precision
// `prec` (BSP_PREC_F64 / F32 / BF16).
int stream_gather(bsp_handle_s* h, const StreamSym& S, int bs, int prec, const double* fvals,
                  const double* dinv, StreamVals& out);

// x = sweep(rhs) on h's stream.  x must hold the sentinel on entry; the
// ticket is reset by this call.  prec selects the value type of `V`.
int stream_sweep(bsp_handle_s* h, const StreamSym& S, int bs, int prec, const StreamVals& V,
                 const double* rhs, double* x, unsigned* ticket);

}  // namespace bsp
