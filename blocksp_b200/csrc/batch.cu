// batch.cu — many independent SPD systems x many right-hand sides, solved by
// block-IChol0 pCG in one CUDA-graph launch on sm_100a.
//
// Reference counterpart: none as a single call.  The reference solves one
// system at a time with IChol0_pCG (blocksp_solvers.hpp:481-492) = pCG
// (:51-105) + IChol0 (blocksp_preconditioners.hpp:364-536); its pCG couples
// the D dims of a solArray<T,B,D> through one alpha/beta, so independent
// right-hand sides mean one IChol0_pCG<T,bs,1> call per system per RHS.  This
// file computes exactly that loop, every (system, RHS) pair with its own
// alpha, beta and stopping test (the reference's mixed rule: first residual
// ||M^-1 b||, then the recursive ||r||), all pairs at once.
//
// Design:
//   * systems of the same block size form a group, stored as ONE block-diagonal
//     BSR matrix (systems concatenated); IChol0 of a block-diagonal matrix is
//     the block-diagonal of the per-system factors, so the existing level /
//     chain analysis and factorisation run once over the whole group, and the
//     sync-free sweeps run every system's chains in the same persistent launch;
//   * right-hand sides are interleaved per block row (the solArray<T,bs,R>
//     layout), so each matrix / factor block is read once for all R of them;
//   * per-pair scalars come from segmented reductions over fixed 64-row tiles
//     that never cross a system: one warp per tile, then one warp per system
//     sums its tiles in tile order, so results do not depend on launch shape;
//   * one pCG iteration of every group (groups run on forked streams) is
//     captured as a CUDA graph; the loop is a device-side `while` conditional
//     node whose condition the last kernel of each iteration sets, so the whole
//     solve is one graph launch with no host round trip (a host-driven replay
//     of the same iteration graph is kept as the alternative mode);
//   * converged systems drop out: every tile, task and reduction of a system
//     whose pairs are all finished is skipped;
//   * launch shapes (threads per CTA and CTAs per SM of the tile kernels, CTAs
//     per SM of the sweeps) are chosen per group by timing the candidates on
//     the group's own data the first time it is solved (an autotuner).
#include <algorithm>
#include <chrono>
#include <cstring>
#include <functional>
#include <numeric>
#include <vector>
#include "precond.hpp"
#include "sentinel.cuh"

namespace bsp {

constexpr int kTileRows = 64;
constexpr int kBatchMaxThreads = 512;
constexpr int kBatchMaxGroups = 4;
enum { BT_RUNNING = 0, BT_CONVERGED = 1, BT_MAXIT = 2, BT_NAN = 4 };

// Per (system, RHS) solver state.
struct BState {
  double rz, alpha, beta, res, tol;
  int done, it, n_hist, pad;
};
struct BOpts {
  double tol;
  int max_iters;
  int pad;
};

// Device view of one group.
struct BGroupP {
  int n_sys, n_tiles;
  const int* tile_sys;      // local system of each tile
  const int* tile_row;      // first row of each tile (rows end at the tile or the system)
  const int64_t* sys_row;   // first row of each system (n_sys + 1)
  const int* sys_tile;      // first tile of each system (n_sys + 1)
  const int* row_ptr;
  const int* col_idx;
  const double* vals;
  double *x, *r, *z, *w, *p, *q, *part0, *part1;
  BState* st;
  int* sys_active;
  unsigned* tickets;        // [0] forward sweep, [1] backward sweep
  double* hist;
  int hist_cap;
  const BOpts* opts;
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Tiles of the group, one warp each (grid-stride over warps).
#define BT_FOR_TILES(g, t)                                                                \
  for (int t = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); t < (g).n_tiles;     \
       t += (int)((gridDim.x * blockDim.x) >> 5))

// ------------------------------------------------------------------ tile kernels
// q = A p for the rows of every active tile; part0 = p . q per tile and RHS.
template <int BS, int R>
__global__ void __launch_bounds__(kBatchMaxThreads) k_bt_spmv(const BGroupP g) {
  using M = BlockMap<BS, double>;
  using CV = typename Chunk<double>::vec;
  constexpr int V = M::V, G = M::G, P = M::P, CPR = M::CPR, RPP = M::RPP, CPB = M::CPB;
  constexpr int RPW = 32 / G;  // rows per warp pass
  constexpr int LD = R * BS;
  const int lane = threadIdx.x & 31, gl = lane % G, grp = lane / G;
  const int c0 = (gl % CPR) * V;
  const CV* vb = reinterpret_cast<const CV*>(g.vals);
  BT_FOR_TILES(g, t) {
    const int s = __ldg(g.tile_sys + t);
    if (!g.sys_active[s]) continue;
    const int r0 = __ldg(g.tile_row + t);
    const int r1 = (int)min((int64_t)r0 + kTileRows, g.sys_row[s + 1]);
    double dot[R];
#pragma unroll
    for (int r = 0; r < R; ++r) dot[r] = 0.0;
    for (int base = r0; base < r1; base += RPW) {
      const int row = base + grp;
      const bool valid = row < r1;
      double acc[P][R];
#pragma unroll
      for (int q = 0; q < P; ++q)
#pragma unroll
        for (int r = 0; r < R; ++r) acc[q][r] = 0.0;
      if (valid) {
        const int beg = __ldg(g.row_ptr + row), end = __ldg(g.row_ptr + row + 1);
        for (int e0 = beg; e0 < end; e0 += 4) {
          CV a[4][P];
          int cols[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            if (e0 + u < end) {
              cols[u] = __ldg(g.col_idx + e0 + u);
#pragma unroll
              for (int q = 0; q < P; ++q) a[u][q] = ld_stream(vb + (int64_t)(e0 + u) * CPB + q * G + gl);
            }
          }
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            if (e0 + u < end) {
#pragma unroll
              for (int r = 0; r < R; ++r) {
                double xv[V];
                ld_vec<V>(g.p + (int64_t)cols[u] * LD + r * BS + c0, xv);
#pragma unroll
                for (int q = 0; q < P; ++q) {
                  double av[V];
                  unpack(a[u][q], av);
#pragma unroll
                  for (int v = 0; v < V; ++v) acc[q][r] = fma(av[v], xv[v], acc[q][r]);
                }
              }
            }
          }
        }
      }
#pragma unroll
      for (int q = 0; q < P; ++q)
#pragma unroll
        for (int r = 0; r < R; ++r) acc[q][r] = row_reduce<CPR>(acc[q][r], 0xffffffffu);
      if (valid && gl % CPR == 0) {
#pragma unroll
        for (int q = 0; q < P; ++q) {
          const int rc = q * RPP + gl / CPR;
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const int64_t k = (int64_t)row * LD + r * BS + rc;
            g.q[k] = acc[q][r];
            dot[r] = fma(g.p[k], acc[q][r], dot[r]);
          }
        }
      }
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const double v = warp_sum(dot[r]);
      if (lane == 0) g.part0[(int64_t)t * R + r] = v;
    }
  }
}

// Element loop over the rows of a tile: lane-strided over the row-major
// [row][RHS][component] range; `rhs` is the RHS index of element e.
#define BT_FOR_ELEMS(e, rhs, r0, r1)                                                  \
  for (int64_t e = (int64_t)(r0) * (R * BS) + (threadIdx.x & 31), _e1 = (int64_t)(r1) * (R * BS); \
       e < _e1; e += 32)                                                              \
    if (const int rhs = (int)((e / BS) % R); true)

template <int R> __device__ __forceinline__ void load_pair_state(const BGroupP& g, int s, bool (&run)[R],
                                                                 double (&a)[R], bool alpha) {
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const BState& S = g.st[s * R + r];
    run[r] = S.done == BT_RUNNING;
    a[r] = alpha ? S.alpha : S.beta;
  }
}
template <int R> __device__ __forceinline__ void pick(const bool (&run)[R], const double (&a)[R], int rhs,
                                                      bool& go, double& av) {
  go = false;
  av = 0.0;
#pragma unroll
  for (int k = 0; k < R; ++k)
    if (k == rhs) {
      go = run[k];
      av = a[k];
    }
}
template <int R> __device__ __forceinline__ void store_partials(double* part, int t, double (&acc)[R]) {
#pragma unroll
  for (int k = 0; k < R; ++k) {
    const double v = warp_sum(acc[k]);
    if ((threadIdx.x & 31) == 0) part[(int64_t)t * R + k] = v;
  }
}

// x += alpha p, r -= alpha q for running pairs; part1 = r . r; the sweep
// outputs w, z of the tile are re-filled with the sentinel.
template <int BS, int R>
__global__ void __launch_bounds__(kBatchMaxThreads) k_bt_update(const BGroupP g) {
  BT_FOR_TILES(g, t) {
    const int s = __ldg(g.tile_sys + t);
    if (!g.sys_active[s]) continue;
    const int r0 = __ldg(g.tile_row + t);
    const int r1 = (int)min((int64_t)r0 + kTileRows, g.sys_row[s + 1]);
    bool run[R];
    double al[R], acc[R];
    load_pair_state<R>(g, s, run, al, true);
#pragma unroll
    for (int k = 0; k < R; ++k) acc[k] = 0.0;
    BT_FOR_ELEMS(e, rhs, r0, r1) {
      bool go;
      double a;
      pick<R>(run, al, rhs, go, a);
      double rv = g.r[e];
      if (go) {
        g.x[e] = fma(a, g.p[e], g.x[e]);
        rv = fma(-a, g.q[e], rv);
        g.r[e] = rv;
      }
      const double sq = rv * rv;
#pragma unroll
      for (int k = 0; k < R; ++k) acc[k] += (k == rhs) ? sq : 0.0;
      reinterpret_cast<unsigned long long*>(g.w)[e] = kSentinel64;
      reinterpret_cast<unsigned long long*>(g.z)[e] = kSentinel64;
    }
    store_partials<R>(g.part1, t, acc);
  }
}

// part0 = r . z per tile and RHS.
template <int BS, int R>
__global__ void __launch_bounds__(kBatchMaxThreads) k_bt_dot_rz(const BGroupP g) {
  BT_FOR_TILES(g, t) {
    const int s = __ldg(g.tile_sys + t);
    if (!g.sys_active[s]) continue;
    const int r0 = __ldg(g.tile_row + t);
    const int r1 = (int)min((int64_t)r0 + kTileRows, g.sys_row[s + 1]);
    double acc[R];
#pragma unroll
    for (int k = 0; k < R; ++k) acc[k] = 0.0;
    BT_FOR_ELEMS(e, rhs, r0, r1) {
      const double v = g.r[e] * g.z[e];
#pragma unroll
      for (int k = 0; k < R; ++k) acc[k] += (k == rhs) ? v : 0.0;
    }
    store_partials<R>(g.part0, t, acc);
  }
}

// p = z + beta p for running pairs.
template <int BS, int R>
__global__ void __launch_bounds__(kBatchMaxThreads) k_bt_pupd(const BGroupP g) {
  BT_FOR_TILES(g, t) {
    const int s = __ldg(g.tile_sys + t);
    if (!g.sys_active[s]) continue;
    const int r0 = __ldg(g.tile_row + t);
    const int r1 = (int)min((int64_t)r0 + kTileRows, g.sys_row[s + 1]);
    bool run[R];
    double be[R];
    load_pair_state<R>(g, s, run, be, false);
    BT_FOR_ELEMS(e, rhs, r0, r1) {
      bool go;
      double b;
      pick<R>(run, be, rhs, go, b);
      if (go) g.p[e] = fma(b, g.p[e], g.z[e]);
    }
  }
}

// Start of a solve: x = 0 and the sweep outputs filled with the sentinel
// (r already holds b).
template <int BS, int R>
__global__ void __launch_bounds__(kBatchMaxThreads) k_bt_init(const BGroupP g) {
  BT_FOR_TILES(g, t) {
    const int s = __ldg(g.tile_sys + t);
    const int r0 = __ldg(g.tile_row + t);
    const int r1 = (int)min((int64_t)r0 + kTileRows, g.sys_row[s + 1]);
    BT_FOR_ELEMS(e, rhs, r0, r1) {
      (void)rhs;
      g.x[e] = 0.0;
      reinterpret_cast<unsigned long long*>(g.w)[e] = kSentinel64;
      reinterpret_cast<unsigned long long*>(g.z)[e] = kSentinel64;
    }
  }
}

// p = z; part0 = z . z (the first residual ||M^-1 b||), part1 = r . z.
template <int BS, int R>
__global__ void __launch_bounds__(kBatchMaxThreads) k_bt_init_dots(const BGroupP g) {
  BT_FOR_TILES(g, t) {
    const int s = __ldg(g.tile_sys + t);
    const int r0 = __ldg(g.tile_row + t);
    const int r1 = (int)min((int64_t)r0 + kTileRows, g.sys_row[s + 1]);
    double a[R], b[R];
#pragma unroll
    for (int k = 0; k < R; ++k) a[k] = b[k] = 0.0;
    BT_FOR_ELEMS(e, rhs, r0, r1) {
      const double zv = g.z[e];
      g.p[e] = zv;
      const double zz = zv * zv, rz = g.r[e] * zv;
#pragma unroll
      for (int k = 0; k < R; ++k) {
        a[k] += (k == rhs) ? zz : 0.0;
        b[k] += (k == rhs) ? rz : 0.0;
      }
    }
    store_partials<R>(g.part0, t, a);
    store_partials<R>(g.part1, t, b);
  }
}

// ------------------------------------------------------------------ per-pair scalars
enum { FIN_INIT = 0, FIN_ALPHA = 1, FIN_RES = 2, FIN_BETA = 3 };

// One warp per system: sums the system's tile partials in tile order, then
// updates the state of each of its R pairs (solvers.hpp:57-97).
template <int R, int MODE>
__global__ void k_bt_fin(const BGroupP g) {
  const int s = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (MODE == FIN_RES && blockIdx.x == 0 && threadIdx.x < 2) g.tickets[threadIdx.x] = 0u;
  if (s >= g.n_sys) return;
  if (MODE != FIN_INIT && !g.sys_active[s]) return;
  const int t0 = g.sys_tile[s], t1 = g.sys_tile[s + 1];
  const double* src = (MODE == FIN_RES) ? g.part1 : g.part0;
  double a[R], b[R];
#pragma unroll
  for (int k = 0; k < R; ++k) a[k] = b[k] = 0.0;
  for (int t = t0 + lane; t < t1; t += 32) {
#pragma unroll
    for (int k = 0; k < R; ++k) {
      a[k] += src[(int64_t)t * R + k];
      if (MODE == FIN_INIT) b[k] += g.part1[(int64_t)t * R + k];
    }
  }
#pragma unroll
  for (int k = 0; k < R; ++k) {
    a[k] = warp_sum(a[k]);
    if (MODE == FIN_INIT) b[k] = warp_sum(b[k]);
  }
  if (lane != 0) return;
  const double tol = g.opts->tol;
  const int max_iters = g.opts->max_iters;
  int any = 0;
#pragma unroll
  for (int k = 0; k < R; ++k) {
    BState& S = g.st[s * R + k];
    double* hist = g.hist ? g.hist + (int64_t)(s * R + k) * g.hist_cap : nullptr;
    if (MODE == FIN_INIT) {
      // res_mag[0] = ||M^-1 b||, tolerance = res_mag[0] * tol (solvers.hpp:57-66)
      const double res0 = sqrt(a[k]);
      S.res = res0;
      S.tol = res0 * tol;
      S.rz = b[k];
      S.alpha = S.beta = 0.0;
      S.it = 0;
      S.n_hist = 1;
      if (hist && g.hist_cap > 0) hist[0] = res0;
      S.done = !isfinite(res0) ? BT_NAN : (res0 > S.tol ? BT_RUNNING : BT_CONVERGED);
    } else if (S.done == BT_RUNNING) {
      if (MODE == FIN_ALPHA) {
        S.alpha = S.rz / a[k];
      } else if (MODE == FIN_RES) {
        const double res = sqrt(a[k]);
        S.res = res;
        if (hist && S.n_hist < g.hist_cap) hist[S.n_hist] = res;
        S.n_hist++;
        if (!isfinite(res)) S.done = BT_NAN;
        else if (!(res > S.tol)) S.done = BT_CONVERGED;
      } else {  // FIN_BETA
        S.beta = a[k] / S.rz;
        S.rz = a[k];
        S.it++;
        if (S.it > max_iters) S.done = BT_MAXIT;
      }
    }
    any |= S.done == BT_RUNNING;
  }
  g.sys_active[s] = any;
}

struct BContP {
  const BState* st[kBatchMaxGroups];
  int n_pairs[kBatchMaxGroups];
  int n_groups;
  int* counter;   // iterations executed
  int* running;   // 1 while any pair runs (read by the host-driven mode)
  int cap;        // hard bound on iterations
  const DevStatus* dev_st;  // device error word: a failed sweep ends the loop
};

// Decides whether another iteration runs; sets the graph's loop condition.
__global__ void k_bt_continue(BContP c, cudaGraphConditionalHandle hnd, int use_cond, int bump) {
  int any = 0;
  for (int gi = 0; gi < c.n_groups; ++gi)
    for (int i = threadIdx.x; i < c.n_pairs[gi]; i += blockDim.x) any |= c.st[gi][i].done == BT_RUNNING;
  any = __syncthreads_or(any);
  if (threadIdx.x == 0) {
    // an iteration counts when the previous decision let it run (a host-driven
    // replay after the end changes nothing)
    const int it = *c.counter + ((bump && *c.running) ? 1 : 0);
    *c.counter = it;
    // a sweep that timed out (or any other device failure) ends the loop at
    // once: the host reads the status after the launch
    const int run = any && it < c.cap && *reinterpret_cast<const volatile int*>(&c.dev_st->code) == 0;
    *c.running = run;
    if (use_cond) cudaGraphSetConditional(hnd, run ? 1u : 0u);
  }
}

// user layout (systems in order, each n_s x R x bs) <-> group layout
__global__ void k_bt_copy(int n_sys, const int64_t* __restrict__ user_off, const int64_t* __restrict__ sys_row,
                          int ld, const double* __restrict__ src, double* __restrict__ dst, int to_group) {
  const int s = blockIdx.y;
  if (s >= n_sys) return;
  const int64_t len = (sys_row[s + 1] - sys_row[s]) * ld;
  const int64_t go = sys_row[s] * ld, uo = user_off[s];
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < len; e += (int64_t)gridDim.x * blockDim.x) {
    if (to_group) dst[go + e] = src[uo + e];
    else dst[uo + e] = src[go + e];
  }
}

// ------------------------------------------------------------------ sweeps
// Multi-RHS sync-free IChol0 sweeps over the chains of every active system.
// TRANS = false: w_i = L_ii^-1 (r_i - sum_{j<i} L_ij w_j)      (forward, L by rows)
// TRANS = true:  z_i = L_ii^-T (w_i - sum_{j>i} L_ji^T z_j)    (backward, L by columns)
// (blocksp_preconditioners.hpp:432-489, per RHS.)
struct BSweepP {
  int n_tasks;
  const int* task_row;
  const int* task_len;
  const int* task_sys;
  int task_dir;
  const int* sys_active;
  const int* ptr;
  const int* idx;
  const int64_t* blk;  // null: entry index
  const int* diag;     // forward: entries [ptr[i], diag[i])
  const double* vals;
  const double* dinv;
  const double* rhs;
  double* x;
  unsigned* ticket;
  DevStatus* st;
  unsigned spin_limit;  // polls before a wait gives up with BSP_TIMEOUT
};

constexpr int kBSweepThreads = 256;

template <int BS, int R, bool TRANS>
__global__ void __launch_bounds__(kBSweepThreads) k_bt_sweep(const BSweepP p) {
  using M = BlockMap<BS, double>;
  using CV = typename Chunk<double>::vec;
  constexpr int V = M::V, G = M::G, P = M::P, CPR = M::CPR, RPP = M::RPP, CPB = M::CPB;
  constexpr int GPC = kBSweepThreads / G;
  constexpr int LD = R * BS;
  // dependency entries whose blocks are loaded ahead: fewer with more RHS,
  // whose x values take the registers
  constexpr int NPF = (P == 1) ? (R >= 4 ? 2 : 4) : (P == 2 && R < 4 ? 2 : 1);
  constexpr int XV = TRANS ? P : V;
  __shared__ double sm_s[GPC][LD];
  __shared__ double sm_x[GPC][LD];
  const int gl = threadIdx.x % G;
  const int gid = threadIdx.x / G;
  const int lane = threadIdx.x & 31;
  const int gbase = lane - gl;
  const unsigned gmask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << gbase);
  const int c0 = (gl % CPR) * V;
  const CV* vb = reinterpret_cast<const CV*>(p.vals);
  double* s = sm_s[gid];
  double* xs = sm_x[gid];
  while (true) {
    int t = 0;
    if (gl == 0) t = (int)atomicAdd(p.ticket, 1u);
    t = __shfl_sync(gmask, t, gbase);
    if (t >= p.n_tasks) break;
    if (!p.sys_active[__ldg(p.task_sys + t)]) continue;
    const int i0 = __ldg(p.task_row + t);
    const int len = __ldg(p.task_len + t);
    CV nf[NPF][P], nd[P];
    int nbeg, nend;
    auto range = [&](int r, int& b0, int& b1) {
      b0 = __ldg(p.ptr + r);
      b1 = TRANS ? __ldg(p.ptr + r + 1) : __ldg(p.diag + r);
    };
    auto prefetch = [&](int r, int& b0, int& b1) {
      range(r, b0, b1);
#pragma unroll
      for (int u = 0; u < NPF; ++u) {
        if (b0 + u < b1) {
          const int64_t b = p.blk ? __ldg(p.blk + b0 + u) : (int64_t)(b0 + u);
#pragma unroll
          for (int q = 0; q < P; ++q) nf[u][q] = ld_stream(vb + b * CPB + q * G + gl);
        }
      }
      const CV* db = reinterpret_cast<const CV*>(p.dinv) + (int64_t)r * CPB;
#pragma unroll
      for (int q = 0; q < P; ++q) nd[q] = ld_stream(db + q * G + gl);
    };
    prefetch(i0, nbeg, nend);
    for (int step = 0; step < len; ++step) {
      const int i = i0 + step * p.task_dir;
      const int prev = step > 0 ? i - p.task_dir : -1;
      const int beg = nbeg, end = nend;
      CV pf[NPF][P], pd[P];
#pragma unroll
      for (int u = 0; u < NPF; ++u)
#pragma unroll
        for (int q = 0; q < P; ++q) pf[u][q] = nf[u][q];
#pragma unroll
      for (int q = 0; q < P; ++q) pd[q] = nd[q];
      if (step + 1 < len) prefetch(i + p.task_dir, nbeg, nend);
      double acc[P][R];   // forward: per block row q and RHS
      double tac[R][V];   // backward: per RHS and column
#pragma unroll
      for (int r = 0; r < R; ++r) {
#pragma unroll
        for (int q = 0; q < P; ++q) acc[q][r] = 0.0;
#pragma unroll
        for (int v = 0; v < V; ++v) tac[r][v] = 0.0;
      }
      // x values of dependency j for every RHS: from shared memory when j is
      // the chain's previous row, else from global memory (polled)
      auto load_x = [&](bool from_prev, int j, double (&xv)[R][XV]) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
          if constexpr (!TRANS) {
            if (from_prev) {
#pragma unroll
              for (int v = 0; v < V; ++v) xv[r][v] = xs[r * BS + c0 + v];
            } else {
              ld_vec_cg<V>(p.x + (int64_t)j * LD + r * BS + c0, xv[r]);
            }
          } else {
#pragma unroll
            for (int q = 0; q < P; ++q) {
              const int rr = q * RPP + gl / CPR;
              xv[r][q] = from_prev ? xs[r * BS + rr] : __ldcg(p.x + (int64_t)j * LD + r * BS + rr);
            }
          }
        }
      };
      auto poll_x = [&](int j, double (&xv)[R][XV]) {
        bool pending = false;
#pragma unroll
        for (int r = 0; r < R; ++r)
#pragma unroll
          for (int v = 0; v < XV; ++v) pending |= is_sentinel(xv[r][v]);
        unsigned spins = 0;
        while (pending) {
          poll_pause(spins);
          pending = false;
#pragma unroll
          for (int r = 0; r < R; ++r) {
#pragma unroll
            for (int v = 0; v < XV; ++v) {
              const int64_t k = TRANS ? (int64_t)j * LD + r * BS + v * RPP + gl / CPR
                                      : (int64_t)j * LD + r * BS + c0 + v;
              xv[r][v] = ld_poll(p.x + k);
              pending |= is_sentinel(xv[r][v]);
            }
          }
          if (pending) {
            if (++spins > p.spin_limit) {
              set_status(p.st, BSP_TIMEOUT, i);
              break;
            }
            if ((spins & 255u) == 0u && *reinterpret_cast<volatile int*>(&p.st->code) != 0) break;
          }
        }
      };
      auto fma_entry = [&](const CV (&a)[P], const double (&xv)[R][XV]) {
#pragma unroll
        for (int q = 0; q < P; ++q) {
          double av[V];
          unpack(a[q], av);
#pragma unroll
          for (int r = 0; r < R; ++r) {
            if constexpr (!TRANS) {
#pragma unroll
              for (int v = 0; v < V; ++v) acc[q][r] = fma(av[v], xv[r][v], acc[q][r]);
            } else {
#pragma unroll
              for (int v = 0; v < V; ++v) tac[r][v] = fma(av[v], xv[r][q], tac[r][v]);
            }
          }
        }
      };
      {
        double xv[NPF][R][XV];
        int jj[NPF];
        bool has[NPF];
#pragma unroll
        for (int u = 0; u < NPF; ++u) {
          has[u] = beg + u < end;
          if (has[u]) {
            jj[u] = __ldg(p.idx + beg + u);
            load_x(jj[u] == prev, jj[u], xv[u]);
          }
        }
#pragma unroll
        for (int u = 0; u < NPF; ++u) {
          if (has[u]) {
            if (jj[u] != prev) poll_x(jj[u], xv[u]);
            fma_entry(pf[u], xv[u]);
          }
        }
      }
      for (int e = beg + NPF; e < end; ++e) {
        const int j = __ldg(p.idx + e);
        const int64_t b = p.blk ? __ldg(p.blk + e) : (int64_t)e;
        CV a[P];
#pragma unroll
        for (int q = 0; q < P; ++q) a[q] = ld_stream(vb + b * CPB + q * G + gl);
        double xv[R][XV];
        load_x(j == prev, j, xv);
        if (j != prev) poll_x(j, xv);
        fma_entry(a, xv);
      }
      // s = rhs_i - sum
      if constexpr (!TRANS) {
#pragma unroll
        for (int q = 0; q < P; ++q)
#pragma unroll
          for (int r = 0; r < R; ++r) acc[q][r] = row_reduce<CPR>(acc[q][r], gmask);
        if (gl % CPR == 0) {
#pragma unroll
          for (int q = 0; q < P; ++q) {
            const int rr = q * RPP + gl / CPR;
#pragma unroll
            for (int r = 0; r < R; ++r)
              s[r * BS + rr] = __ldcg(p.rhs + (int64_t)i * LD + r * BS + rr) - acc[q][r];
          }
        }
      } else {
#pragma unroll
        for (int r = 0; r < R; ++r)
#pragma unroll
          for (int v = 0; v < V; ++v)
#pragma unroll
            for (int o = CPR; o < G; o <<= 1) tac[r][v] += __shfl_xor_sync(gmask, tac[r][v], o);
        if (gl < CPR) {
#pragma unroll
          for (int r = 0; r < R; ++r)
#pragma unroll
            for (int v = 0; v < V; ++v)
              s[r * BS + c0 + v] = __ldcg(p.rhs + (int64_t)i * LD + r * BS + c0 + v) - tac[r][v];
        }
      }
      __syncwarp(gmask);
      if constexpr (!TRANS) {
        // x_i = L_ii^-1 s: lane holds Dinv[row q][c0..c0+V)
#pragma unroll
        for (int q = 0; q < P; ++q) {
          double av[V];
          unpack(pd[q], av);
          double o[R];
#pragma unroll
          for (int r = 0; r < R; ++r) {
            o[r] = 0.0;
#pragma unroll
            for (int v = 0; v < V; ++v) o[r] = fma(av[v], s[r * BS + c0 + v], o[r]);
            o[r] = row_reduce<CPR>(o[r], gmask);
          }
          if (gl % CPR == 0) {
            const int rr = q * RPP + gl / CPR;
#pragma unroll
            for (int r = 0; r < R; ++r) {
              p.x[(int64_t)i * LD + r * BS + rr] = o[r];
              xs[r * BS + rr] = o[r];
            }
          }
        }
      } else {
        // x_i = L_ii^-T s: lane holds Dinv[rr][c0..c0+V) and adds Dinv[rr][c] s[rr]
        double o[R][V];
#pragma unroll
        for (int r = 0; r < R; ++r)
#pragma unroll
          for (int v = 0; v < V; ++v) o[r][v] = 0.0;
#pragma unroll
        for (int q = 0; q < P; ++q) {
          const int rr = q * RPP + gl / CPR;
          double av[V];
          unpack(pd[q], av);
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const double sr = s[r * BS + rr];
#pragma unroll
            for (int v = 0; v < V; ++v) o[r][v] = fma(av[v], sr, o[r][v]);
          }
        }
#pragma unroll
        for (int r = 0; r < R; ++r)
#pragma unroll
          for (int v = 0; v < V; ++v)
#pragma unroll
            for (int off = CPR; off < G; off <<= 1) o[r][v] += __shfl_xor_sync(gmask, o[r][v], off);
        if (gl < CPR) {
#pragma unroll
          for (int r = 0; r < R; ++r)
#pragma unroll
            for (int v = 0; v < V; ++v) {
              p.x[(int64_t)i * LD + r * BS + c0 + v] = o[r][v];
              xs[r * BS + c0 + v] = o[r][v];
            }
        }
      }
      __syncwarp(gmask);
    }
  }
}

}  // namespace bsp

// ================================================================= host side
using namespace bsp;

namespace {

struct TuneCfg {
  int threads = 256, ctas_per_sm = 2;   // tile kernels
  int sweep_ctas_per_sm = 0;            // 0: occupancy maximum
};

struct BatchGroup {
  int bs = 0;
  std::vector<int> sys;            // global ids of the group's systems
  std::vector<int64_t> row_off;    // first row of each system (n_sys + 1)
  bsp_matrix_t A = nullptr;
  bsp_precond_t pc = nullptr;
  int n_tiles = 0;
  DevBuf<int> tile_sys, tile_row, sys_tile, task_sys_lo, task_sys_up;
  DevBuf<int64_t> sys_row, user_off;
  // per-solve state for R right-hand sides
  int R = 0, hist_cap = 0;
  DevBuf<double> x, r, z, w, p, q, part0, part1, hist;
  DevBuf<BState> st;
  DevBuf<int> sys_active;
  DevBuf<unsigned> tickets;
  TuneCfg tune;
  bool tuned = false;
  int n_sys() const { return (int)sys.size(); }
  int64_t n_rows() const { return row_off.back(); }
};

}  // namespace

struct bsp_batch_s {
  bsp_handle_t h = nullptr;
  int device = 0;
  int n_sys = 0;
  std::vector<int> n_rows, bs;
  std::vector<int> group_of, local_of;  // per system
  std::vector<BatchGroup> groups;
  DevBuf<BOpts> opts;
  DevBuf<int> counter;  // [0] iterations, [1] running
  cudaStream_t cap = nullptr;
  cudaStream_t gs[kBatchMaxGroups] = {};
  cudaEvent_t fork = nullptr, join[kBatchMaxGroups] = {};
  // cached graphs (valid for graph_R / graph_hist / graph_mode)
  cudaGraphExec_t exec = nullptr, exec_body = nullptr;
  int graph_R = 0, graph_hist = -1, graph_mode = -1;
  int64_t init_kernels = 0, body_kernels = 0;
  ~bsp_batch_s() {
    if (exec) cudaGraphExecDestroy(exec);
    if (exec_body) cudaGraphExecDestroy(exec_body);
    for (auto& g : groups) {
      if (g.pc) bsp_precond_destroy(g.pc);
      if (g.A) bsp_matrix_destroy(g.A);
    }
    for (int i = 0; i < kBatchMaxGroups; ++i) {
      if (gs[i]) cudaStreamDestroy(gs[i]);
      if (join[i]) cudaEventDestroy(join[i]);
    }
    if (fork) cudaEventDestroy(fork);
    if (cap) cudaStreamDestroy(cap);
  }
};

namespace {

int grid_of(const bsp_batch_s* B, int ctas_per_sm) { return std::max(1, B->h->num_sms * ctas_per_sm); }

BGroupP view(bsp_batch_s* B, BatchGroup& g) {
  BGroupP v{};
  v.n_sys = g.n_sys();
  v.n_tiles = g.n_tiles;
  v.tile_sys = g.tile_sys.get();
  v.tile_row = g.tile_row.get();
  v.sys_row = g.sys_row.get();
  v.sys_tile = g.sys_tile.get();
  v.row_ptr = g.A->row_ptr.get();
  v.col_idx = g.A->col_idx.get();
  v.vals = g.A->vals.get();
  v.x = g.x.get();
  v.r = g.r.get();
  v.z = g.z.get();
  v.w = g.w.get();
  v.p = g.p.get();
  v.q = g.q.get();
  v.part0 = g.part0.get();
  v.part1 = g.part1.get();
  v.st = g.st.get();
  v.sys_active = g.sys_active.get();
  v.tickets = g.tickets.get();
  v.hist = g.hist_cap > 0 ? g.hist.get() : nullptr;
  v.hist_cap = g.hist_cap;
  v.opts = B->opts.get();
  return v;
}

BSweepP sweep_params(bsp_batch_s* B, BatchGroup& g, bool fwd) {
  bsp_precond_s* pc = g.pc;
  BSweepP p{};
  p.sys_active = g.sys_active.get();
  p.dinv = pc->dinv.get();
  p.vals = pc->f_vals.get();
  p.st = B->h->ws.status.get();
  p.spin_limit = B->h->spin_limit;
  if (fwd) {
    p.n_tasks = pc->n_task_lo;
    p.task_row = pc->task_lo_row.get();
    p.task_len = pc->task_lo_len.get();
    p.task_sys = g.task_sys_lo.get();
    p.task_dir = 1;
    p.ptr = pc->f_ptr.get();
    p.idx = pc->f_col.get();
    p.diag = pc->f_diag.get();
    p.blk = nullptr;
    p.rhs = g.r.get();
    p.x = g.w.get();
    p.ticket = g.tickets.get();
  } else {
    p.n_tasks = pc->n_task_up;
    p.task_row = pc->task_up_row.get();
    p.task_len = pc->task_up_len.get();
    p.task_sys = g.task_sys_up.get();
    p.task_dir = -1;
    p.ptr = pc->t_ptr.get();
    p.idx = pc->t_row.get();
    p.blk = pc->t_blk.get();
    p.diag = nullptr;
    p.rhs = g.w.get();
    p.x = g.z.get();
    p.ticket = g.tickets.get() + 1;
  }
  return p;
}

// Kernel set of one (block size, R) instantiation.
struct Kernels {
  void (*spmv)(const BGroupP);
  void (*update)(const BGroupP);
  void (*dot_rz)(const BGroupP);
  void (*pupd)(const BGroupP);
  void (*init)(const BGroupP);
  void (*init_dots)(const BGroupP);
  void (*fin_init)(const BGroupP);
  void (*fin_alpha)(const BGroupP);
  void (*fin_res)(const BGroupP);
  void (*fin_beta)(const BGroupP);
  void (*sweep_fwd)(const BSweepP);
  void (*sweep_bwd)(const BSweepP);
};

template <int BS, int R> Kernels kernels_t() {
  return Kernels{k_bt_spmv<BS, R>,        k_bt_update<BS, R>,      k_bt_dot_rz<BS, R>,
                 k_bt_pupd<BS, R>,        k_bt_init<BS, R>,        k_bt_init_dots<BS, R>,
                 k_bt_fin<R, FIN_INIT>,   k_bt_fin<R, FIN_ALPHA>,  k_bt_fin<R, FIN_RES>,
                 k_bt_fin<R, FIN_BETA>,   k_bt_sweep<BS, R, false>, k_bt_sweep<BS, R, true>};
}

template <int BS> bool kernels_r(int R, Kernels& k) {
  switch (R) {
    case 1: k = kernels_t<BS, 1>(); return true;
    case 2: k = kernels_t<BS, 2>(); return true;
    case 4: k = kernels_t<BS, 4>(); return true;
    default: return false;
  }
}

bool kernels_for(int bs, int R, Kernels& k) {
  switch (bs) {
    case 4: return kernels_r<4>(R, k);
    case 8: return kernels_r<8>(R, k);
    case 16: return kernels_r<16>(R, k);
    default: return false;
  }
}

int sweep_grid(bsp_batch_s* B, BatchGroup& g, void (*kern)(const BSweepP)) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBSweepThreads, 0) != cudaSuccess || per_sm < 1) {
    cudaGetLastError();
    per_sm = 1;
  }
  if (g.tune.sweep_ctas_per_sm > 0) per_sm = std::min(per_sm, g.tune.sweep_ctas_per_sm);
  return grid_of(B, per_sm);
}

// Enqueues the kernels of one phase of one group; returns the number of kernels.
int enqueue_group(bsp_batch_s* B, BatchGroup& g, const Kernels& k, cudaStream_t s, bool init) {
  const BGroupP v = view(B, g);
  const int tg = grid_of(B, g.tune.ctas_per_sm), tt = g.tune.threads;
  const int fin_grid = (g.n_sys() * 32 + 255) / 256;
  const BSweepP fw = sweep_params(B, g, true), bw = sweep_params(B, g, false);
  const int sg_f = sweep_grid(B, g, k.sweep_fwd), sg_b = sweep_grid(B, g, k.sweep_bwd);
  if (init) {
    k.init<<<tg, tt, 0, s>>>(v);
    cudaMemsetAsync(g.sys_active.get(), 1, g.n_sys() * sizeof(int), s);
    cudaMemsetAsync(g.tickets.get(), 0, 2 * sizeof(unsigned), s);
    k.sweep_fwd<<<sg_f, kBSweepThreads, 0, s>>>(fw);
    k.sweep_bwd<<<sg_b, kBSweepThreads, 0, s>>>(bw);
    k.init_dots<<<tg, tt, 0, s>>>(v);
    k.fin_init<<<fin_grid, 256, 0, s>>>(v);
    return 5;
  }
  k.spmv<<<tg, tt, 0, s>>>(v);
  k.fin_alpha<<<fin_grid, 256, 0, s>>>(v);
  k.update<<<tg, tt, 0, s>>>(v);
  k.fin_res<<<fin_grid, 256, 0, s>>>(v);  // also zeroes the sweep tickets
  k.sweep_fwd<<<sg_f, kBSweepThreads, 0, s>>>(fw);
  k.sweep_bwd<<<sg_b, kBSweepThreads, 0, s>>>(bw);
  k.dot_rz<<<tg, tt, 0, s>>>(v);
  k.fin_beta<<<fin_grid, 256, 0, s>>>(v);
  k.pupd<<<tg, tt, 0, s>>>(v);
  return 9;
}

BContP cont_params(bsp_batch_s* B, int max_iters) {
  BContP c{};
  c.n_groups = (int)B->groups.size();
  for (int i = 0; i < c.n_groups; ++i) {
    c.st[i] = B->groups[i].st.get();
    c.n_pairs[i] = B->groups[i].n_sys() * B->groups[i].R;
  }
  c.counter = B->counter.get();
  c.running = B->counter.get() + 1;
  c.cap = max_iters + 2;
  c.dev_st = B->h->ws.status.get();
  return c;
}

// Fork the phase over the group streams and join back into `s`.
int enqueue_phase(bsp_batch_s* B, const std::vector<Kernels>& ks, cudaStream_t s, bool init,
                  cudaGraphConditionalHandle hnd, int use_cond, int max_iters) {
  int n = 0;
  BSP_CUDA_TRY(cudaEventRecord(B->fork, s));
  for (size_t gi = 0; gi < B->groups.size(); ++gi) {
    BSP_CUDA_TRY(cudaStreamWaitEvent(B->gs[gi], B->fork, 0));
    n += enqueue_group(B, B->groups[gi], ks[gi], B->gs[gi], init);
    BSP_CUDA_TRY(cudaEventRecord(B->join[gi], B->gs[gi]));
    BSP_CUDA_TRY(cudaStreamWaitEvent(s, B->join[gi], 0));
  }
  k_bt_continue<<<1, 256, 0, s>>>(cont_params(B, max_iters), hnd, use_cond, init ? 0 : 1);
  BSP_CUDA_TRY(cudaPeekAtLastError());
  return n + 1;
}

int alloc_state(bsp_batch_s* B, BatchGroup& g, int R, int hist_cap) {
  if (g.R != R) {
    const size_t nv = (size_t)g.n_rows() * R * g.bs;
    for (DevBuf<double>* v : {&g.x, &g.r, &g.z, &g.w, &g.p, &g.q}) {
      BSP_TRY(v->alloc(nv));
      BSP_CUDA_TRY(cudaMemset(v->get(), 0, nv * sizeof(double)));
    }
    BSP_TRY(g.part0.alloc((size_t)g.n_tiles * R));
    BSP_TRY(g.part1.alloc((size_t)g.n_tiles * R));
    BSP_TRY(g.st.alloc((size_t)g.n_sys() * R));
    BSP_CUDA_TRY(cudaMemset(g.st.get(), 0, (size_t)g.n_sys() * R * sizeof(BState)));
    // user offsets of the group's systems for this R
    std::vector<int64_t> all(B->n_sys + 1, 0), uo(g.n_sys());
    for (int s = 0; s < B->n_sys; ++s) all[s + 1] = all[s] + (int64_t)B->n_rows[s] * B->bs[s] * R;
    for (int i = 0; i < g.n_sys(); ++i) uo[i] = all[g.sys[i]];
    BSP_TRY(g.user_off.alloc(uo.size()));
    BSP_CUDA_TRY(cudaMemcpy(g.user_off.get(), uo.data(), uo.size() * sizeof(int64_t), cudaMemcpyHostToDevice));
    g.R = R;
    g.hist_cap = -1;
  }
  if (g.hist_cap != hist_cap) {
    if (hist_cap > 0) BSP_TRY(g.hist.alloc((size_t)g.n_sys() * R * hist_cap));
    else g.hist.release();
    g.hist_cap = hist_cap;
  }
  return BSP_OK;
}

float time_ms(cudaStream_t s, const std::function<void()>& f, int reps) {
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  f();  // warm-up
  cudaEventRecord(a, s);
  for (int i = 0; i < reps; ++i) f();
  cudaEventRecord(b, s);
  cudaEventSynchronize(b);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return ms / reps;
}

// Autotuner: time each candidate launch shape on the group's own data.  The
// candidates compute identical results (reductions are per fixed tile, sweep
// rows do not depend on scheduling), so only speed differs.
int autotune(bsp_batch_s* B, BatchGroup& g, const Kernels& k) {
  cudaStream_t s = B->cap;
  BSP_CUDA_TRY(cudaMemsetAsync(g.sys_active.get(), 1, g.n_sys() * sizeof(int), s));
  BSP_CUDA_TRY(cudaMemsetAsync(g.st.get(), 0, (size_t)g.n_sys() * g.R * sizeof(BState), s));
  const BGroupP v = view(B, g);
  float best = 1e30f;
  TuneCfg bestc = g.tune;
  for (int threads : {128, 256, 512}) {
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k.spmv, threads, 0);
    for (int cps : {1, 2, 4, 8}) {
      if (cps > std::max(occ, 1)) continue;
      const int grid = grid_of(B, cps);
      const float ms = time_ms(s, [&] { k.spmv<<<grid, threads, 0, s>>>(v); }, 3);
      bsp::count_launch_add(4);
      if (ms < best) {
        best = ms;
        bestc.threads = threads;
        bestc.ctas_per_sm = cps;
      }
    }
  }
  g.tune.threads = bestc.threads;
  g.tune.ctas_per_sm = bestc.ctas_per_sm;
  // sweeps: CTAs per SM of the persistent grid
  int occ = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k.sweep_fwd, kBSweepThreads, 0);
  occ = std::max(occ, 1);
  const BSweepP fw = sweep_params(B, g, true);
  best = 1e30f;
  int best_sw = occ;
  for (int cps : {1, 2, 4, 8}) {
    if (cps > occ) continue;
    const int grid = grid_of(B, cps);
    const float ms = time_ms(s, [&] {
      k.init<<<grid_of(B, g.tune.ctas_per_sm), g.tune.threads, 0, s>>>(v);
      cudaMemsetAsync(g.tickets.get(), 0, sizeof(unsigned), s);
      k.sweep_fwd<<<grid, kBSweepThreads, 0, s>>>(fw);
    }, 3);
    bsp::count_launch_add(8);
    if (ms < best) {
      best = ms;
      best_sw = cps;
    }
  }
  g.tune.sweep_ctas_per_sm = best_sw;
  g.tuned = true;
  BSP_CUDA_TRY(cudaStreamSynchronize(s));
  BSP_CUDA_TRY(cudaPeekAtLastError());
  return BSP_OK;
}

void destroy_graphs(bsp_batch_s* B) {
  if (B->exec) cudaGraphExecDestroy(B->exec);
  if (B->exec_body) cudaGraphExecDestroy(B->exec_body);
  B->exec = B->exec_body = nullptr;
  B->graph_R = 0;
}

// Captures the solve.  mode 0: init + while(body) in one graph; mode 1: init
// and body as two graphs, the body replayed by the host.
int build_graphs(bsp_batch_s* B, const std::vector<Kernels>& ks, int mode, int max_iters) {
  destroy_graphs(B);
  cudaStream_t s = B->cap;
  if (mode == 0) {
    cudaGraph_t graph = nullptr, init = nullptr;
    BSP_CUDA_TRY(cudaGraphCreate(&graph, 0));
    cudaGraphConditionalHandle hnd;
    // the loop body runs at least once; from then on its last kernel decides
    BSP_CUDA_TRY(cudaGraphConditionalHandleCreate(&hnd, graph, 1, cudaGraphCondAssignDefault));
    BSP_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
    B->init_kernels = enqueue_phase(B, ks, s, true, hnd, 0, max_iters);
    BSP_CUDA_TRY(cudaStreamEndCapture(s, &init));
    cudaGraphNode_t init_node, cond_node;
    BSP_CUDA_TRY(cudaGraphAddChildGraphNode(&init_node, graph, nullptr, 0, init));
    cudaGraphDestroy(init);
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = hnd;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    BSP_CUDA_TRY(cudaGraphAddNode(&cond_node, graph, &init_node, 1, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    BSP_CUDA_TRY(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    B->body_kernels = enqueue_phase(B, ks, s, false, hnd, 1, max_iters);
    BSP_CUDA_TRY(cudaStreamEndCapture(s, &body));
    const cudaError_t e = cudaGraphInstantiate(&B->exec, graph, 0);
    cudaGraphDestroy(graph);
    BSP_CUDA_TRY(e);
  } else {
    cudaGraph_t init = nullptr, body = nullptr;
    BSP_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
    B->init_kernels = enqueue_phase(B, ks, s, true, 0, 0, max_iters);
    BSP_CUDA_TRY(cudaStreamEndCapture(s, &init));
    BSP_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
    B->body_kernels = enqueue_phase(B, ks, s, false, 0, 0, max_iters);
    BSP_CUDA_TRY(cudaStreamEndCapture(s, &body));
    cudaError_t e = cudaGraphInstantiate(&B->exec, init, 0);
    if (e == cudaSuccess) e = cudaGraphInstantiate(&B->exec_body, body, 0);
    cudaGraphDestroy(init);
    cudaGraphDestroy(body);
    BSP_CUDA_TRY(e);
  }
  return BSP_OK;
}

}  // namespace

// ================================================================= C ABI
extern "C" {

int bsp_batch_create(bsp_handle_t h, int n_sys, const int* n_rows, const int* bs, const int64_t* nnzb,
                     const int* row_ptr, const int* col_idx, const double* vals, bsp_batch_t* out) {
  if (!h || !out || n_sys < 1 || n_sys > 65535 || !n_rows || !bs || !nnzb || !row_ptr || !col_idx || !vals)
    return BSP_INVALID;
  *out = nullptr;
  BSP_CUDA_TRY(cudaSetDevice(h->device));
  auto B = std::make_unique<bsp_batch_s>();
  B->h = h;
  B->device = h->device;
  B->n_sys = n_sys;
  B->n_rows.assign(n_rows, n_rows + n_sys);
  B->bs.assign(bs, bs + n_sys);
  B->group_of.resize(n_sys);
  B->local_of.resize(n_sys);
  // offsets of each system in the packed inputs
  std::vector<int64_t> rp_off(n_sys + 1, 0), ci_off(n_sys + 1, 0), v_off(n_sys + 1, 0);
  for (int s = 0; s < n_sys; ++s) {
    if (n_rows[s] < 1 || nnzb[s] < 0 || (bs[s] != 4 && bs[s] != 8 && bs[s] != 16)) {
      record_error("batched systems need n_rows >= 1 and block size 4, 8 or 16");
      return BSP_INVALID;
    }
    rp_off[s + 1] = rp_off[s] + n_rows[s] + 1;
    ci_off[s + 1] = ci_off[s] + nnzb[s];
    v_off[s + 1] = v_off[s] + nnzb[s] * (int64_t)bs[s] * bs[s];
  }
  // groups by block size, systems in input order
  std::vector<int> sizes;
  for (int s = 0; s < n_sys; ++s)
    if (std::find(sizes.begin(), sizes.end(), bs[s]) == sizes.end()) sizes.push_back(bs[s]);
  std::sort(sizes.begin(), sizes.end());
  B->groups.resize(sizes.size());
  for (size_t gi = 0; gi < sizes.size(); ++gi) {
    BatchGroup& g = B->groups[gi];
    g.bs = sizes[gi];
    g.row_off.push_back(0);
    for (int s = 0; s < n_sys; ++s)
      if (bs[s] == g.bs) {
        B->group_of[s] = (int)gi;
        B->local_of[s] = g.n_sys();
        g.sys.push_back(s);
        g.row_off.push_back(g.row_off.back() + n_rows[s]);
      }
    const int64_t nr = g.n_rows();
    int64_t nnz_g = 0;
    for (int s : g.sys) nnz_g += nnzb[s];
    if (nr > (int64_t)INT32_MAX / 2 || nnz_g > (int64_t)INT32_MAX) {
      record_error("a batched group exceeds 32-bit block indices");
      return BSP_INVALID;
    }
    // block-diagonal concatenation
    std::vector<int> grp(nr + 1), gci(nnz_g);
    int64_t e = 0;
    for (int i = 0; i < g.n_sys(); ++i) {
      const int s = g.sys[i];
      const int ro = (int)g.row_off[i];
      const int* rp = row_ptr + rp_off[s];
      if (rp[0] != 0 || rp[n_rows[s]] != nnzb[s]) {
        record_error("batched system row pointers must start at 0 and end at nnzb");
        return BSP_INVALID;
      }
      for (int r = 0; r < n_rows[s]; ++r) grp[ro + r] = (int)(e + rp[r]);
      const int* ci = col_idx + ci_off[s];
      for (int64_t k = 0; k < nnzb[s]; ++k) {
        if (ci[k] < 0 || ci[k] >= n_rows[s]) {
          record_error("batched system column index out of range");
          return BSP_INVALID;
        }
        gci[e + k] = ci[k] + ro;
      }
      e += nnzb[s];
    }
    grp[nr] = (int)e;
    BSP_TRY(matrix_create_struct(h, (int)nr, (int)nr, g.bs, nnz_g, grp.data(), gci.data(), &g.A));
    {
      int64_t off = 0;
      for (int s : g.sys) {
        const size_t n = (size_t)nnzb[s] * g.bs * g.bs;
        if (n) BSP_CUDA_TRY(cudaMemcpy(g.A->vals.get() + off, vals + v_off[s], n * sizeof(double), cudaMemcpyHostToDevice));
        off += (int64_t)n;
      }
    }
    bsp_precond_params pp{};
    pp.kind = BSP_PC_ICHOL0;
    pp.precision = BSP_PREC_F64;
    BSP_TRY(bsp_precond_create(h, g.A, &pp, &g.pc));
    // tiles (never crossing a system) and the system of each sweep task
    std::vector<int> tsys, trow, stile(g.n_sys() + 1, 0);
    for (int i = 0; i < g.n_sys(); ++i) {
      stile[i] = (int)tsys.size();
      for (int64_t r = g.row_off[i]; r < g.row_off[i + 1]; r += kTileRows) {
        tsys.push_back(i);
        trow.push_back((int)r);
      }
    }
    stile[g.n_sys()] = (int)tsys.size();
    g.n_tiles = (int)tsys.size();
    auto up = [](auto& d, const auto& v) -> int {
      BSP_TRY(d.alloc(v.size()));
      BSP_CUDA_TRY(cudaMemcpy(d.get(), v.data(), v.size() * sizeof(v[0]), cudaMemcpyHostToDevice));
      return BSP_OK;
    };
    BSP_TRY(up(g.tile_sys, tsys));
    BSP_TRY(up(g.tile_row, trow));
    BSP_TRY(up(g.sys_tile, stile));
    BSP_TRY(up(g.sys_row, g.row_off));
    for (int lower = 1; lower >= 0; --lower) {
      const int nt = lower ? g.pc->n_task_lo : g.pc->n_task_up;
      std::vector<int> rows(std::max(nt, 1)), ts(std::max(nt, 1), 0);
      if (nt)
        BSP_CUDA_TRY(cudaMemcpy(rows.data(), lower ? g.pc->task_lo_row.get() : g.pc->task_up_row.get(),
                                nt * sizeof(int), cudaMemcpyDeviceToHost));
      for (int t = 0; t < nt; ++t)
        ts[t] = (int)(std::upper_bound(g.row_off.begin(), g.row_off.end(), (int64_t)rows[t]) - g.row_off.begin()) - 1;
      BSP_TRY(up(lower ? g.task_sys_lo : g.task_sys_up, ts));
    }
    BSP_TRY(g.sys_active.alloc(g.n_sys()));
    BSP_TRY(g.tickets.alloc(2));
    BSP_CUDA_TRY(cudaMemset(g.tickets.get(), 0, 2 * sizeof(unsigned)));
  }
  BSP_TRY(B->opts.alloc(1));
  BSP_TRY(B->counter.alloc(2));
  BSP_CUDA_TRY(cudaStreamCreateWithFlags(&B->cap, cudaStreamNonBlocking));
  for (size_t gi = 0; gi < B->groups.size(); ++gi) {
    BSP_CUDA_TRY(cudaStreamCreateWithFlags(&B->gs[gi], cudaStreamNonBlocking));
    BSP_CUDA_TRY(cudaEventCreateWithFlags(&B->join[gi], cudaEventDisableTiming));
  }
  BSP_CUDA_TRY(cudaEventCreateWithFlags(&B->fork, cudaEventDisableTiming));
  BSP_CUDA_TRY(cudaDeviceSynchronize());
  *out = B.release();
  return BSP_OK;
}

int bsp_batch_destroy(bsp_batch_t B) {
  if (!B) return BSP_OK;
  cudaSetDevice(B->device);
  delete B;
  return BSP_OK;
}

int bsp_batch_tuning(bsp_batch_t B, int* n_groups, int* group_bs, int* group_systems, int64_t* group_rows,
                     int* tile_threads, int* tile_ctas_per_sm, int* sweep_ctas_per_sm) {
  if (!B) return BSP_INVALID;
  const int ng = (int)B->groups.size();
  if (n_groups) *n_groups = ng;
  for (int i = 0; i < ng; ++i) {
    const BatchGroup& g = B->groups[i];
    if (group_bs) group_bs[i] = g.bs;
    if (group_systems) group_systems[i] = g.n_sys();
    if (group_rows) group_rows[i] = g.n_rows();
    if (tile_threads) tile_threads[i] = g.tuned ? g.tune.threads : 0;
    if (tile_ctas_per_sm) tile_ctas_per_sm[i] = g.tuned ? g.tune.ctas_per_sm : 0;
    if (sweep_ctas_per_sm) sweep_ctas_per_sm[i] = g.tuned ? g.tune.sweep_ctas_per_sm : 0;
  }
  return BSP_OK;
}

int bsp_batch_pcg_dev(bsp_handle_t h, bsp_batch_t B, int nrhs, const double* b, double* x,
                      const bsp_batch_opts* o, bsp_batch_info* info) {
  if (!h || !B || !b || !x || !o || h != B->h) return BSP_INVALID;
  if (nrhs != 1 && nrhs != 2 && nrhs != 4) {
    record_error("batched pCG supports 1, 2 or 4 right-hand sides");
    return BSP_INVALID;
  }
  if (o->max_iters < 0 || !(o->tol >= 0.0) || (o->mode != 0 && o->mode != 1)) return BSP_INVALID;
  BSP_CUDA_TRY(cudaSetDevice(h->device));
  const auto t_setup = std::chrono::steady_clock::now();
  std::vector<Kernels> ks(B->groups.size());
  for (size_t gi = 0; gi < B->groups.size(); ++gi)
    if (!kernels_for(B->groups[gi].bs, nrhs, ks[gi])) return BSP_INVALID;
  const int hist_cap = o->hist_cap > 0 ? o->hist_cap : 0;
  bool rebuild = B->graph_R != nrhs || B->graph_hist != hist_cap || B->graph_mode != o->mode || o->retune;
  for (auto& g : B->groups) {
    if (g.R != nrhs || g.hist_cap != hist_cap) rebuild = true;
    BSP_TRY(alloc_state(B, g, nrhs, hist_cap));
  }
  BSP_CUDA_TRY(cudaStreamSynchronize(h->stream));
  if (rebuild) {
    for (size_t gi = 0; gi < B->groups.size(); ++gi)
      if (!B->groups[gi].tuned || o->retune) BSP_TRY(autotune(B, B->groups[gi], ks[gi]));
    BSP_TRY(build_graphs(B, ks, o->mode, o->max_iters));
    B->graph_R = nrhs;
    B->graph_hist = hist_cap;
    B->graph_mode = o->mode;
  }
  const double setup_ms =
      rebuild ? std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_setup).count() : 0.0;
  EventTimer tm(h->stream);
  BOpts ho{o->tol, o->max_iters, 0};
  BSP_CUDA_TRY(cudaMemcpyAsync(B->opts.get(), &ho, sizeof(BOpts), cudaMemcpyHostToDevice, h->stream));
  BSP_CUDA_TRY(cudaMemsetAsync(B->counter.get(), 0, 2 * sizeof(int), h->stream));
  BSP_CUDA_TRY(cudaMemsetAsync(h->ws.status.get(), 0, sizeof(DevStatus), h->stream));
  for (auto& g : B->groups) {
    dim3 grid(64, g.n_sys());
    bsp::count_launch(), k_bt_copy<<<grid, 256, 0, h->stream>>>(g.n_sys(), g.user_off.get(), g.sys_row.get(),
                                                               nrhs * g.bs, b, g.r.get(), 1);
  }
  BSP_CUDA_TRY(cudaPeekAtLastError());
  int graph_iters = 0;
  BSP_CUDA_TRY(cudaGraphLaunch(B->exec, h->stream));
  if (o->mode == 0) {
    BSP_CUDA_TRY(cudaMemcpyAsync(&graph_iters, B->counter.get(), sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    BSP_CUDA_TRY(cudaStreamSynchronize(h->stream));
  } else {
    const int every = std::max(1, o->check_every);
    int ctr[2] = {0, 1};
    int64_t launches = 0;
    BSP_CUDA_TRY(cudaMemcpyAsync(ctr, B->counter.get(), 2 * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    BSP_CUDA_TRY(cudaStreamSynchronize(h->stream));
    while (ctr[1]) {
      for (int i = 0; i < every; ++i) BSP_CUDA_TRY(cudaGraphLaunch(B->exec_body, h->stream));
      launches += every;
      BSP_CUDA_TRY(cudaMemcpyAsync(ctr, B->counter.get(), 2 * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
      BSP_CUDA_TRY(cudaStreamSynchronize(h->stream));
    }
    graph_iters = ctr[0];
    bsp::count_launch_add(B->init_kernels + B->body_kernels * launches);
  }
  // kernels replayed by the graph (its loop body runs at least once)
  if (o->mode == 0) bsp::count_launch_add(B->init_kernels + B->body_kernels * (int64_t)std::max(graph_iters, 1));
  for (auto& g : B->groups) {
    dim3 grid(64, g.n_sys());
    bsp::count_launch(), k_bt_copy<<<grid, 256, 0, h->stream>>>(g.n_sys(), g.user_off.get(), g.sys_row.get(),
                                                               nrhs * g.bs, g.x.get(), x, 0);
  }
  BSP_CUDA_TRY(cudaPeekAtLastError());
  const double solve_ms = tm.stop_ms();
  DevStatus ds{};
  BSP_CUDA_TRY(cudaMemcpy(&ds, h->ws.status.get(), sizeof(DevStatus), cudaMemcpyDeviceToHost));
  // summary over pairs
  int worst = BSP_OK, iters_max = 0, n_conv = 0, n_pairs = 0;
  int64_t iters_total = 0;
  for (auto& g : B->groups) {
    std::vector<BState> st((size_t)g.n_sys() * nrhs);
    BSP_CUDA_TRY(cudaMemcpy(st.data(), g.st.get(), st.size() * sizeof(BState), cudaMemcpyDeviceToHost));
    n_pairs += (int)st.size();
    for (const BState& S : st) {
      iters_max = std::max(iters_max, S.it);
      iters_total += S.it;
      if (S.done == BT_CONVERGED) ++n_conv;
      const int code = S.done == BT_CONVERGED ? BSP_OK : S.done == BT_NAN ? BSP_NAN : BSP_MAXIT;
      if (worst == BSP_OK) worst = code;
    }
  }
  if (ds.code != 0) {
    record_error("batched sweep reported device status " + std::to_string(ds.code));
    worst = ds.code;
  }
  if (info) {
    info->status = worst;
    info->n_pairs = n_pairs;
    info->n_converged = n_conv;
    info->iters_max = iters_max;
    info->iters_total = iters_total;
    info->graph_iters = graph_iters;
    info->setup_ms = setup_ms;
    info->solve_ms = solve_ms;
  }
  return worst;
}

int bsp_batch_results(bsp_batch_t B, int nrhs, int* iters, int* state, double* final_res, double* hist,
                      int hist_cap) {
  if (!B) return BSP_INVALID;
  for (auto& g : B->groups)
    if (g.R != nrhs) return BSP_INVALID;
  cudaSetDevice(B->device);
  for (auto& g : B->groups) {
    const int ns = g.n_sys();
    std::vector<BState> st((size_t)ns * nrhs);
    BSP_CUDA_TRY(cudaMemcpy(st.data(), g.st.get(), st.size() * sizeof(BState), cudaMemcpyDeviceToHost));
    std::vector<double> hh;
    if (hist && hist_cap > 0 && g.hist_cap > 0) {
      hh.resize((size_t)ns * nrhs * g.hist_cap);
      BSP_CUDA_TRY(cudaMemcpy(hh.data(), g.hist.get(), hh.size() * sizeof(double), cudaMemcpyDeviceToHost));
    }
    for (int i = 0; i < ns; ++i)
      for (int r = 0; r < nrhs; ++r) {
        const BState& S = st[(size_t)i * nrhs + r];
        const size_t o = (size_t)g.sys[i] * nrhs + r;
        if (iters) iters[o] = S.it;
        if (state) state[o] = S.done;
        if (final_res) final_res[o] = S.res;
        if (!hh.empty()) {
          double* dst = hist + o * hist_cap;
          for (int k = 0; k < hist_cap; ++k)
            dst[k] = (k < std::min(S.n_hist, g.hist_cap)) ? hh[((size_t)i * nrhs + r) * g.hist_cap + k] : 0.0;
        }
      }
  }
  return BSP_OK;
}

int bsp_batch_pcg(bsp_handle_t h, bsp_batch_t B, int nrhs, const double* b_host, double* x_host,
                  const bsp_batch_opts* o, bsp_batch_info* info) {
  if (!h || !B || !b_host || !x_host) return BSP_INVALID;
  BSP_CUDA_TRY(cudaSetDevice(h->device));
  size_t n = 0;
  for (int s = 0; s < B->n_sys; ++s) n += (size_t)B->n_rows[s] * B->bs[s] * nrhs;
  BSP_TRY(h->stage(n, n));
  BSP_CUDA_TRY(cudaMemcpyAsync(h->stage_in.get(), b_host, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  const int st = bsp_batch_pcg_dev(h, B, nrhs, h->stage_in.get(), h->stage_out.get(), o, info);
  if (st != BSP_OK && st != BSP_MAXIT && st != BSP_NAN) return st;
  BSP_CUDA_TRY(cudaMemcpyAsync(x_host, h->stage_out.get(), n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  BSP_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return st;
}

}  // extern "C"
