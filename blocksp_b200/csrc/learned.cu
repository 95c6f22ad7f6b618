// learned.cu — learned block preconditioner: a message-passing network over
// the block graph of A, with hand-written forward and backward kernels, trained
// on the GPU, whose output corrects the block-ILU0 factors (LU form, for
// pGMRES) or the block-IChol0 factor (L L^T form, for pCG on SPD systems).
//
// No reference counterpart: the reference's preconditioners end at IChol0
// (blocksp_preconditioners.hpp:364-538).  The factors keep A's sparsity and
// are stored in the ILU0 structures (PC_LEARNED_LU), so the same sync-free
// triangular sweeps apply them (ILU0::invmul order, :294-349).
//
// Network (8x8 blocks, hidden H = 32, 3 layers; nodes = block rows, one
// directed edge per off-diagonal block A_ij in CSR order):
//   s_i = rms(A_ii); x_i = [A_ii / s_i, log s_i]; a_k = A_ij / sqrt(s_i s_j)
//   h = relu(Wn x + bn); e = relu(We a + be)
//   per layer: msg_k = relu(Wm [h_j; e_k] + bm); m_i = sum_{k in row i} msg_k;
//              h_i += relu(Wu [h_i; m_i] + bu)
//   dF_ij = 0.01 c_ij (Wo [h_i; h_j; e_k] + bo);  dF_ii = 0.01 s_i (Wd h_i + bd)
//   with c_ij = sqrt(s_i s_j) for upper blocks (U_ij ~ A_ij) and sqrt(s_i / s_j)
//   for lower blocks (L_ij ~ A_ij U_jj^-1)
// M = L U with (L, U) the ILU0 factors plus dF.  Training minimises the
// left-preconditioned operator's distance from the identity on probes,
//   loss = (1/K) sum_k ||M^-1 A q_k - q_k||^2,
// q_k the orthonormal Arnoldi vectors of the ILU0-preconditioned operator
// started from M0^-1 b (the Krylov basis pGMRES itself builds); its gradient
// needs M^-1 and M^-T, both applied by the sync-free triangular sweeps.
//
// Kernels: every layer is "one warp per row (node or edge), one lane per
// output unit" with the weights transposed into shared memory; they are
// gather/HBM-bound (a few hundred bytes and ~2-6 kflop per row), so they run
// on the FP32 (or FP64) pipes.  Weight gradients are per-CTA partial sums of
// outer products over a fixed partition of the rows, summed in CTA order:
// training steps are deterministic.  Everything is templated on T: float for
// training and inference, double for the gradient check against the oracle.
#include <algorithm>
#include <cmath>
#include <memory>
#include <vector>
#include "precond.hpp"
#include "reduce.cuh"

namespace bsp {
int bsmv_launch(bsp_matrix_s* A, int nrhs, int transpose, int dtype, double alpha, const void* x, double beta,
                const void* z, void* y, cudaStream_t s);
int precond_build_learned(bsp_precond_s* pc, const double* dF);

namespace lf {

constexpr int H = 32;
constexpr int kLayers = 3;
constexpr double kAlpha = 0.01;
constexpr int kB2 = 64;              // 8x8 blocks
constexpr int kWarps = 8;            // warps per CTA of the row kernels
constexpr int kGradBlocks = 2 * kB200SMs;

struct Graph {
  int n, E, nnzb;
  const int* row_ptr;
  const int* col_idx;
  const int* diag_pos;  // n
  const int* e_blk;     // E
  const int* e_row;
  const int* e_col;
  const int* er_ptr;    // n+1: edges of row i
  const int* ec_ptr;    // n+1: edges whose column is j ...
  const int* ec_idx;    // ... listed here by increasing row
};

template <typename T> __device__ __forceinline__ T relu(T v) { return v > T(0) ? v : T(0); }

// Output scale of the correction of block (i, j).  LU form: the scale of U_ij
// for j > i, of L_ij = A_ij U_jj^-1 for j < i.  L L^T form (llt): the scale of
// L_ij = A_ij L_jj^-T, sqrt(s_i), for j < i; upper blocks are not part of L
// (scale 0, so they get neither an output nor a gradient).
template <typename T> __device__ __forceinline__ T edge_scale(const T* s, int i, int j, int llt) {
  const T si = s[i], sj = s[j];
  if (llt) return j < i ? T(kAlpha) * sqrt(si) : T(0);
  return T(kAlpha) * (j < i ? sqrt(si / sj) : sqrt(si * sj));
}
// Diagonal-block scale: s_i (U_ii ~ A_ii) or sqrt(s_i) (L_ii ~ A_ii^1/2).
template <typename T> __device__ __forceinline__ T diag_scale(const T* s, int i, int llt) {
  return T(kAlpha) * (llt ? sqrt(s[i]) : s[i]);
}
// L L^T form: the diagonal correction is lower triangular (L_ii stays a
// triangular factor), entry o = r * 8 + c of the row-major block.
__device__ __forceinline__ bool diag_kept(int o, int llt) { return !llt || (o % 8) <= (o / 8); }

// ------------------------------------------------------------------ row kernels
// out(r, o) = sum_t W[o][t] in_r[t] + b[o], o < NOUT: one warp per row.
template <typename T, int NIN, int NOUT, class In, class Out>
__global__ void __launch_bounds__(kWarps * 32) k_dense(int rows, const T* __restrict__ W,
                                                       const T* __restrict__ bias, In in, Out out) {
  extern __shared__ __align__(16) unsigned char smraw[];
  T* Wt = reinterpret_cast<T*>(smraw);  // [NIN][NOUT]
  T* bs = Wt + NIN * NOUT;
  T* xin = bs + NOUT;                   // [kWarps][NIN]
  for (int e = threadIdx.x; e < NIN * NOUT; e += blockDim.x) {
    const int o = e / NIN, t = e % NIN;
    Wt[t * NOUT + o] = W[e];
  }
  for (int o = threadIdx.x; o < NOUT; o += blockDim.x) bs[o] = bias[o];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  T* xv = xin + warp * NIN;
  for (int r = blockIdx.x * kWarps + warp; r < rows; r += gridDim.x * kWarps) {
    in.load(r, xv, lane);
    __syncwarp();
#pragma unroll
    for (int oo = 0; oo < NOUT / 32; ++oo) {
      const int o = lane + 32 * oo;
      T acc = bs[o];
#pragma unroll 8
      for (int t = 0; t < NIN; ++t) acc = fma(Wt[t * NOUT + o], xv[t], acc);
      out.store(r, o, acc);
    }
    __syncwarp();
  }
}

// out(r, t) = sum_o W[o][t] g_r[o], t < NIN (the input gradient of a layer).
template <typename T, int NIN, int NOUT, class G, class Out>
__global__ void __launch_bounds__(kWarps * 32) k_dense_t(int rows, const T* __restrict__ W, G g, Out out) {
  extern __shared__ __align__(16) unsigned char smraw[];
  T* Ws = reinterpret_cast<T*>(smraw);  // [NOUT][NIN] as stored
  T* gin = Ws + NIN * NOUT;             // [kWarps][NOUT]
  for (int e = threadIdx.x; e < NIN * NOUT; e += blockDim.x) Ws[e] = W[e];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  T* gv = gin + warp * NOUT;
  for (int r = blockIdx.x * kWarps + warp; r < rows; r += gridDim.x * kWarps) {
    g.load(r, gv, lane);
    __syncwarp();
#pragma unroll
    for (int tt = 0; tt < (NIN + 31) / 32; ++tt) {
      const int t = lane + 32 * tt;
      if (t < NIN) {
        T acc = T(0);
#pragma unroll 8
        for (int o = 0; o < NOUT; ++o) acc = fma(Ws[o * NIN + t], gv[o], acc);
        out.store(r, t, acc);
      }
    }
    __syncwarp();
  }
}

// Partial weight/bias gradients: CTA b sums g_r in_r^T and g_r over its fixed
// chunk of rows; part[b][NOUT*NIN + NOUT].
template <typename T, int NIN, int NOUT, class G, class In>
__global__ void __launch_bounds__(256) k_wgrad(int rows, G g, In in, T* __restrict__ part) {
  constexpr int NE = NOUT * NIN + NOUT;
  constexpr int PER = (NE + 255) / 256;
  constexpr int RB = 16;
  __shared__ T sg[RB][NOUT];
  __shared__ T sx[RB][NIN];
  T acc[PER];
#pragma unroll
  for (int p = 0; p < PER; ++p) acc[p] = T(0);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int chunk = (rows + gridDim.x - 1) / gridDim.x;
  const int r0 = blockIdx.x * chunk, r1 = min(rows, r0 + chunk);
  for (int base = r0; base < r1; base += RB) {
    for (int q = warp; q < RB; q += 8) {
      const int r = base + q;
      if (r < r1) {
        g.load(r, sg[q], lane);
        in.load(r, sx[q], lane);
      } else {
        for (int o = lane; o < NOUT; o += 32) sg[q][o] = T(0);
        for (int t = lane; t < NIN; t += 32) sx[q][t] = T(0);
      }
    }
    __syncthreads();
#pragma unroll
    for (int p = 0; p < PER; ++p) {
      const int e = threadIdx.x + p * 256;
      if (e < NOUT * NIN) {
        const int o = e / NIN, t = e % NIN;
        T s = T(0);
#pragma unroll
        for (int q = 0; q < RB; ++q) s = fma(sg[q][o], sx[q][t], s);
        acc[p] += s;
      } else if (e < NE) {
        const int o = e - NOUT * NIN;
        T s = T(0);
#pragma unroll
        for (int q = 0; q < RB; ++q) s += sg[q][o];
        acc[p] += s;
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int p = 0; p < PER; ++p) {
    const int e = threadIdx.x + p * 256;
    if (e < NE) part[(int64_t)blockIdx.x * NE + e] = acc[p];
  }
}

template <typename T>
__global__ void k_wgrad_sum(int ne, int nb, const T* __restrict__ part, T* __restrict__ out) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  T s = T(0);
  for (int b = 0; b < nb; ++b) s += part[(int64_t)b * ne + e];
  out[e] = s;
}

// ------------------------------------------------------------------ features
template <typename T>
__global__ void k_node_features(Graph g, const double* __restrict__ vals, T* __restrict__ s, T* __restrict__ x) {
  const int lane = threadIdx.x & 31;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < g.n; i += (gridDim.x * blockDim.x) >> 5) {
    const double* D = vals + (int64_t)g.diag_pos[i] * kB2;
    T ss = T(0);
    for (int c = lane; c < kB2; c += 32) ss += T(D[c]) * T(D[c]);
    for (int o = 16; o > 0; o >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, o);
    const T si = sqrt(ss / T(kB2));
    T* xi = x + (int64_t)i * (kB2 + 1);
    for (int c = lane; c < kB2; c += 32) xi[c] = T(D[c]) / si;
    if (lane == 0) {
      xi[kB2] = log(si);
      s[i] = si;
    }
  }
}

template <typename T>
__global__ void k_edge_features(Graph g, const double* __restrict__ vals, const T* __restrict__ s,
                                T* __restrict__ a) {
  const int lane = threadIdx.x & 31;
  for (int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < g.E; k += (gridDim.x * blockDim.x) >> 5) {
    const double* B = vals + (int64_t)g.e_blk[k] * kB2;
    const T den = sqrt(s[g.e_row[k]] * s[g.e_col[k]]);
    for (int c = lane; c < kB2; c += 32) a[(int64_t)k * kB2 + c] = T(B[c]) / den;
  }
}

// ------------------------------------------------------------------ functors
// Input rows (each loads NIN values into dst with the 32 lanes of a warp).
template <typename T, int N> struct RowIn {       // dst = src[r]
  const T* src;
  __device__ void load(int r, T* dst, int lane) const {
    for (int t = lane; t < N; t += 32) dst[t] = src[(int64_t)r * N + t];
  }
};
template <typename T> struct MsgIn {               // [h[col(k)]; e[k]]
  const T* h;
  const T* e;
  const int* col;
  __device__ void load(int k, T* dst, int lane) const {
    dst[lane] = h[(int64_t)col[k] * H + lane];
    dst[H + lane] = e[(int64_t)k * H + lane];
  }
};
template <typename T> struct UpdIn {               // [h[i]; m[i]], m summed here and stored
  const T* h;
  const T* msg;
  const int* er_ptr;
  T* m;
  __device__ void load(int i, T* dst, int lane) const {
    T acc = T(0);
    for (int k = er_ptr[i]; k < er_ptr[i + 1]; ++k) acc += msg[(int64_t)k * H + lane];
    m[(int64_t)i * H + lane] = acc;
    dst[lane] = h[(int64_t)i * H + lane];
    dst[H + lane] = acc;
  }
};
template <typename T> struct UpdInStored {         // [h[i]; m[i]] with m already stored
  const T* h;
  const T* m;
  __device__ void load(int i, T* dst, int lane) const {
    dst[lane] = h[(int64_t)i * H + lane];
    dst[H + lane] = m[(int64_t)i * H + lane];
  }
};
template <typename T> struct DecIn {               // [h[row]; h[col]; e[k]]
  const T* h;
  const T* e;
  const int* row;
  const int* col;
  __device__ void load(int k, T* dst, int lane) const {
    dst[lane] = h[(int64_t)row[k] * H + lane];
    dst[H + lane] = h[(int64_t)col[k] * H + lane];
    dst[2 * H + lane] = e[(int64_t)k * H + lane];
  }
};

// Outputs
template <typename T> struct ReluOut {
  T* dst;
  __device__ void store(int r, int o, T v) const { dst[(int64_t)r * H + o] = relu(v); }
};
template <typename T> struct ResidOut {            // u = relu(v); h_next = h + u
  const T* h;
  T* u;
  T* hn;
  __device__ void store(int r, int o, T v) const {
    const T uv = relu(v);
    u[(int64_t)r * H + o] = uv;
    hn[(int64_t)r * H + o] = h[(int64_t)r * H + o] + uv;
  }
};
template <typename T> struct DecEdgeOut {          // dF[blk] = edge_scale v
  const T* s;
  const int* row;
  const int* col;
  const int* blk;
  double* dF;
  int llt;
  __device__ void store(int k, int o, T v) const {
    dF[(int64_t)blk[k] * kB2 + o] = double(edge_scale(s, row[k], col[k], llt) * v);
  }
};
template <typename T> struct DecDiagOut {
  const T* s;
  const int* diag;
  double* dF;
  int llt;
  __device__ void store(int i, int o, T v) const {
    dF[(int64_t)diag[i] * kB2 + o] = diag_kept(o, llt) ? double(diag_scale(s, i, llt) * v) : 0.0;
  }
};

// Gradient rows
template <typename T> struct GEdgeDec {            // edge_scale gdF[blk[k]]
  const T* s;
  const int* row;
  const int* col;
  const int* blk;
  const T* gdF;
  int llt;
  __device__ void load(int k, T* dst, int lane) const {
    const T sc = edge_scale(s, row[k], col[k], llt);
    for (int o = lane; o < kB2; o += 32) dst[o] = sc * gdF[(int64_t)blk[k] * kB2 + o];
  }
};
template <typename T> struct GDiagDec {
  const T* s;
  const int* diag;
  const T* gdF;
  int llt;
  __device__ void load(int i, T* dst, int lane) const {
    const T sc = diag_scale(s, i, llt);
    for (int o = lane; o < kB2; o += 32)
      dst[o] = diag_kept(o, llt) ? sc * gdF[(int64_t)diag[i] * kB2 + o] : T(0);
  }
};
template <typename T> struct GMask {               // g[r] * (act[r] > 0)
  const T* g;
  const T* act;
  __device__ void load(int r, T* dst, int lane) const {
    const T a = act[(int64_t)r * H + lane];
    dst[lane] = a > T(0) ? g[(int64_t)r * H + lane] : T(0);
  }
};
template <typename T> struct GMaskRow {            // dm[row(k)] * (msg[k] > 0)
  const T* dm;
  const T* msg;
  const int* row;
  __device__ void load(int k, T* dst, int lane) const {
    const T a = msg[(int64_t)k * H + lane];
    dst[lane] = a > T(0) ? dm[(int64_t)row[k] * H + lane] : T(0);
  }
};

// Input-gradient outputs
template <typename T> struct SplitDecOut {         // t<H: gdr, t<2H: gdc, else de
  T* gdr;
  T* gdc;
  T* de;
  __device__ void store(int k, int t, T v) const {
    if (t < H) gdr[(int64_t)k * H + t] = v;
    else if (t < 2 * H) gdc[(int64_t)k * H + t - H] = v;
    else de[(int64_t)k * H + t - 2 * H] = v;
  }
};
template <typename T> struct DiagDhOut {           // dh[i] = v + sum gdr(row i) + sum gdc(col i)
  Graph g;
  const T* gdr;
  const T* gdc;
  T* dh;
  __device__ void store(int i, int t, T v) const {
    T acc = v;
    for (int k = g.er_ptr[i]; k < g.er_ptr[i + 1]; ++k) acc += gdr[(int64_t)k * H + t];
    for (int q = g.ec_ptr[i]; q < g.ec_ptr[i + 1]; ++q) acc += gdc[(int64_t)g.ec_idx[q] * H + t];
    dh[(int64_t)i * H + t] = acc;
  }
};
template <typename T> struct UpdBwdOut {           // t<H: dh2 = dh + v; else dm
  const T* dh;
  T* dh2;
  T* dm;
  __device__ void store(int i, int t, T v) const {
    if (t < H) dh2[(int64_t)i * H + t] = dh[(int64_t)i * H + t] + v;
    else dm[(int64_t)i * H + t - H] = v;
  }
};
template <typename T> struct MsgBwdOut {           // t<H: gmh; else de += v
  T* gmh;
  T* de;
  __device__ void store(int k, int t, T v) const {
    if (t < H) gmh[(int64_t)k * H + t] = v;
    else de[(int64_t)k * H + t - H] += v;
  }
};

template <typename T>
__global__ void k_gather_cols(Graph g, const T* __restrict__ gmh, T* __restrict__ dh) {
  const int lane = threadIdx.x & 31;
  for (int j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; j < g.n; j += (gridDim.x * blockDim.x) >> 5) {
    T acc = dh[(int64_t)j * H + lane];
    for (int q = g.ec_ptr[j]; q < g.ec_ptr[j + 1]; ++q) acc += gmh[(int64_t)g.ec_idx[q] * H + lane];
    dh[(int64_t)j * H + lane] = acc;
  }
}

// ------------------------------------------------------------------ loss
// loss = (1/K) sum_k ||M^-1 A q_k - q_k||^2 (FP64; probes orthonormal).  With
// z = M^-1 A q, g = (2/K)(z - q), w = U^-T g, lam = L^-T w, y = U z:
//   d loss / d L_ij = -sum_k lam_k[i] y_k[j]^T   (strictly lower blocks)
//   d loss / d U_ij = -sum_k   w_k[i] z_k[j]^T   (upper blocks, diagonal included)
__global__ void k_diff(int64_t n, const double* __restrict__ z, const double* __restrict__ q, double* __restrict__ e) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    e[i] = z[i] - q[i];
}
__global__ void k_scale(int64_t n, double a, double* __restrict__ x) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] *= a;
}
// y = U z over the factor's upper blocks (row-sorted factor structure)
__global__ void k_upper_prod(int n, int bs, const int* __restrict__ fptr, const int* __restrict__ fcol,
                             const int* __restrict__ fdiag, const double* __restrict__ f, const double* __restrict__ z,
                             double* __restrict__ y) {
  const int64_t N = (int64_t)n * bs;
  const int b2 = bs * bs;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < N; e += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(e / bs), r = (int)(e % bs);
    double acc = 0.0;
    for (int b = fdiag[i]; b < fptr[i + 1]; ++b) {
      const int j = fcol[b];
      const double* blk = f + (int64_t)b * b2 + r * bs;
      for (int c = 0; c < bs; ++c) acc = fma(blk[c], z[(int64_t)j * bs + c], acc);
    }
    y[e] = acc;
  }
}
// gradient of every factor block, written in A's block order (perm: factor -> A)
template <typename T>
__global__ void k_factor_grad(int n, int bs, int K, int64_t N, const int* __restrict__ fptr,
                              const int* __restrict__ fcol, const int* __restrict__ fdiag,
                              const int64_t* __restrict__ perm, const double* __restrict__ lam,
                              const double* __restrict__ y, const double* __restrict__ w,
                              const double* __restrict__ z, T* __restrict__ gdF) {
  const int lane = threadIdx.x & 31;
  const int b2 = bs * bs;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += (gridDim.x * blockDim.x) >> 5) {
    for (int b = fptr[i]; b < fptr[i + 1]; ++b) {
      const int j = fcol[b];
      const bool lower = b < fdiag[i];
      const double* left = lower ? lam : w;
      const double* right = lower ? y : z;
      for (int e = lane; e < b2; e += 32) {
        const int r = e / bs, c = e % bs;
        double acc = 0.0;
        for (int k = 0; k < K; ++k)
          acc = fma(left[(int64_t)k * N + (int64_t)i * bs + r], right[(int64_t)k * N + (int64_t)j * bs + c], acc);
        gdF[perm[b] * b2 + e] = T(-acc);
      }
    }
  }
}

// L L^T form.  loss = (1/K) sum_k ||M^-1 A q_k - q_k||^2 with M = L L^T: with
// z = M^-1 A q, g = (2/K)(z - q), w = M^-1 g (M is symmetric), y = L^T z and
// u = L^T w,
//   d loss / d L_ij = -sum_k (w_k[i] y_k[j]^T + z_k[i] u_k[j]^T)   (j <= i)
// y = L^T z over the transposed strictly-lower structure plus the diagonal.
__global__ void k_lower_t_prod(int n, int bs, const int* __restrict__ tptr, const int* __restrict__ trow,
                               const int64_t* __restrict__ tblk, const int* __restrict__ fdiag,
                               const double* __restrict__ f, const double* __restrict__ z, double* __restrict__ y) {
  const int64_t N = (int64_t)n * bs;
  const int b2 = bs * bs;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < N; e += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(e / bs), c = (int)(e % bs);
    double acc = 0.0;
    const double* d = f + (int64_t)fdiag[i] * b2;
    for (int r = 0; r < bs; ++r) acc = fma(d[r * bs + c], z[(int64_t)i * bs + r], acc);
    for (int t = tptr[i]; t < tptr[i + 1]; ++t) {
      const double* blk = f + tblk[t] * b2;  // L_{trow[t], i}
      const int j = trow[t];
      for (int r = 0; r < bs; ++r) acc = fma(blk[r * bs + c], z[(int64_t)j * bs + r], acc);
    }
    y[e] = acc;
  }
}
template <typename T>
__global__ void k_factor_grad_llt(int n, int bs, int K, int64_t N, const int* __restrict__ fptr,
                                  const int* __restrict__ fcol, const int* __restrict__ fdiag,
                                  const int64_t* __restrict__ perm, const double* __restrict__ w,
                                  const double* __restrict__ y, const double* __restrict__ z,
                                  const double* __restrict__ u, T* __restrict__ gdF) {
  const int lane = threadIdx.x & 31;
  const int b2 = bs * bs;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += (gridDim.x * blockDim.x) >> 5) {
    for (int b = fptr[i]; b < fptr[i + 1]; ++b) {
      const int j = fcol[b];
      const bool diag = b == fdiag[i];
      for (int e = lane; e < b2; e += 32) {
        const int r = e / bs, c = e % bs;
        double acc = 0.0;
        if (!diag || c <= r)
          for (int k = 0; k < K; ++k) {
            const int64_t oi = (int64_t)k * N + (int64_t)i * bs + r, oj = (int64_t)k * N + (int64_t)j * bs + c;
            acc = fma(w[oi], y[oj], acc);
            acc = fma(z[oi], u[oj], acc);
          }
        gdF[perm[b] * b2 + e] = T(-acc);
      }
    }
  }
}

template <typename T>
__global__ void k_adam(int64_t n, T* __restrict__ p, const T* __restrict__ g, T* __restrict__ m, T* __restrict__ v,
                       T lr, T b1, T b2, T eps, T c1, T c2) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const T gi = g[i];
    const T mi = b1 * m[i] + (T(1) - b1) * gi;
    const T vi = b2 * v[i] + (T(1) - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrt(vi / c2) + eps);
  }
}

template <typename T> __global__ void k_cast(int64_t n, const double* __restrict__ a, T* __restrict__ b) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = T(a[i]);
}

// F0 in A's block order from the ILU0 factor order: F0[perm[e]] = f[e]
__global__ void k_scatter_f0(int64_t nblk, int b2, const int64_t* __restrict__ perm, const double* __restrict__ f,
                             double* __restrict__ F0) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nblk * b2; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t blk = e / b2, c = e % b2;
    F0[perm[blk] * b2 + c] = f[e];
  }
}

__global__ void k_normalize(int64_t n, const double* __restrict__ v, const double* __restrict__ nrm2,
                            double* __restrict__ q) {
  const double s = 1.0 / sqrt(*nrm2);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    q[i] = v[i] * s;
}
__global__ void k_sub_one(int64_t n, const double* __restrict__ t, double* __restrict__ v) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    v[i] -= t[i];
}
__global__ void k_sub_proj(int64_t n, const double* __restrict__ a, const double* __restrict__ x,
                           double* __restrict__ y) {
  const double s = -*a;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = fma(s, x[i], y[i]);
}

}  // namespace lf
}  // namespace bsp

// ================================================================= host side
using namespace bsp;
using namespace bsp::lf;

namespace {

struct ParamSlot {
  int64_t off;  // W offset; the bias follows W
  int nout, nin;
};

struct GraphBuf {
  const bsp_matrix_s* A = nullptr;
  DevBuf<int> diag_pos, e_blk, e_row, e_col, er_ptr, ec_ptr, ec_idx;
  int n = 0, E = 0;
  Graph view() const {
    Graph g{};
    g.n = n;
    g.E = E;
    g.nnzb = (int)A->nnzb;
    g.row_ptr = A->row_ptr.get();
    g.col_idx = A->col_idx.get();
    g.diag_pos = diag_pos.get();
    g.e_blk = e_blk.get();
    g.e_row = e_row.get();
    g.e_col = e_col.get();
    g.er_ptr = er_ptr.get();
    g.ec_ptr = ec_ptr.get();
    g.ec_idx = ec_idx.get();
    return g;
  }
};

template <typename V> int upload_vec(DevBuf<V>& d, const std::vector<V>& v) {
  BSP_TRY(d.alloc(std::max<size_t>(v.size(), 1)));
  if (!v.empty()) BSP_CUDA_TRY(cudaMemcpy(d.get(), v.data(), v.size() * sizeof(V), cudaMemcpyHostToDevice));
  return BSP_OK;
}

int build_graph(const bsp_matrix_s* A, GraphBuf& G) {
  const int n = A->n_rows;
  const auto& rp = A->h_row_ptr;
  const auto& ci = A->h_col_idx;
  std::vector<int> diag(n, -1), eb, er, ec, erp(n + 1, 0);
  for (int i = 0; i < n; ++i) {
    for (int b = rp[i]; b < rp[i + 1]; ++b) {
      if (ci[b] == i) {
        diag[i] = b;
      } else {
        eb.push_back(b);
        er.push_back(i);
        ec.push_back(ci[b]);
      }
    }
    erp[i + 1] = (int)eb.size();
    if (diag[i] < 0) {
      record_error("learned preconditioner: block row " + std::to_string(i) + " has no diagonal block");
      return BSP_INVALID;
    }
  }
  const int E = (int)eb.size();
  // edges by column, rows increasing (stable counting sort)
  std::vector<int> ecp(n + 1, 0), eci(E);
  for (int k = 0; k < E; ++k) ecp[ec[k] + 1]++;
  for (int j = 0; j < n; ++j) ecp[j + 1] += ecp[j];
  {
    std::vector<int> fill(ecp.begin(), ecp.end() - 1);
    for (int k = 0; k < E; ++k) eci[fill[ec[k]]++] = k;
  }
  G.A = A;
  G.n = n;
  G.E = E;
  BSP_TRY(upload_vec(G.diag_pos, diag));
  BSP_TRY(upload_vec(G.e_blk, eb));
  BSP_TRY(upload_vec(G.e_row, er));
  BSP_TRY(upload_vec(G.e_col, ec));
  BSP_TRY(upload_vec(G.er_ptr, erp));
  BSP_TRY(upload_vec(G.ec_ptr, ecp));
  BSP_TRY(upload_vec(G.ec_idx, eci));
  return BSP_OK;
}

struct ModelBase {
  virtual ~ModelBase() = default;
  virtual int forward(bsp_handle_s* h, const bsp_matrix_s* A, double* dF) = 0;
  virtual int loss_grad(bsp_handle_s* h, const bsp_matrix_s* A, const bsp_precond_s* ilu, int K,
                        const double* probes, double* loss) = 0;
  virtual int adam(bsp_handle_s* h, double lr, double b1, double b2, double eps) = 0;
  virtual int get(double* out, int64_t cnt, int which) = 0;
  virtual int set(const double* in, int64_t cnt) = 0;
  // true while both decoders are exactly zero (the network's output dF is zero)
  virtual bool decoders_zero() const = 0;
};

}  // namespace

struct bsp_learned_s {
  bsp_handle_t h = nullptr;
  int device = 0;
  int bs = 0, dtype = 0;
  int form = BSP_LEARNED_LU;  // factor form the network emits
  double relax = 0.0;        // off-diagonal factor blocks scaled by 1 + relax
  int64_t n_params = 0;
  std::vector<ParamSlot> slots;
  std::unique_ptr<ModelBase> impl;
};

namespace {

std::vector<ParamSlot> layout(int64_t& total) {
  std::vector<ParamSlot> s;
  int64_t off = 0;
  auto add = [&](int nout, int nin) {
    s.push_back({off, nout, nin});
    off += (int64_t)nout * nin + nout;
  };
  add(H, kB2 + 1);  // Wn, bn
  add(H, kB2);      // We, be
  for (int l = 0; l < kLayers; ++l) {
    add(H, 2 * H);  // Wm_l, bm_l
    add(H, 2 * H);  // Wu_l, bu_l
  }
  add(kB2, 3 * H);  // Wo, bo
  add(kB2, H);      // Wd, bd
  total = off;
  return s;
}

template <typename T, int NIN, int NOUT, class In, class Out>
int run_dense(bsp_handle_s* h, int rows, const T* W, const T* b, In in, Out out) {
  if (rows <= 0) return BSP_OK;
  const size_t smem = (size_t)(NIN * NOUT + NOUT + kWarps * NIN) * sizeof(T);
  auto kern = k_dense<T, NIN, NOUT, In, Out>;
  BSP_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int grid = (int)std::min<int64_t>(ceil_div(rows, kWarps), (int64_t)h->num_sms * 8);
  bsp::count_launch(), kern<<<grid, kWarps * 32, smem, h->stream>>>(rows, W, b, in, out);
  BSP_CUDA_TRY(cudaPeekAtLastError());
  return BSP_OK;
}

template <typename T, int NIN, int NOUT, class G, class Out>
int run_dense_t(bsp_handle_s* h, int rows, const T* W, G g, Out out) {
  if (rows <= 0) return BSP_OK;
  const size_t smem = (size_t)(NIN * NOUT + kWarps * NOUT) * sizeof(T);
  auto kern = k_dense_t<T, NIN, NOUT, G, Out>;
  BSP_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int grid = (int)std::min<int64_t>(ceil_div(rows, kWarps), (int64_t)h->num_sms * 8);
  bsp::count_launch(), kern<<<grid, kWarps * 32, smem, h->stream>>>(rows, W, g, out);
  BSP_CUDA_TRY(cudaPeekAtLastError());
  return BSP_OK;
}

template <typename T, int NIN, int NOUT, class G, class In>
int run_wgrad(bsp_handle_s* h, int rows, G g, In in, T* part, T* out) {
  constexpr int NE = NOUT * NIN + NOUT;
  bsp::count_launch(), k_wgrad<T, NIN, NOUT, G, In><<<kGradBlocks, 256, 0, h->stream>>>(rows, g, in, part);
  bsp::count_launch(), k_wgrad_sum<T><<<(NE + 255) / 256, 256, 0, h->stream>>>(NE, kGradBlocks, part, out);
  BSP_CUDA_TRY(cudaPeekAtLastError());
  return BSP_OK;
}

// grow-only allocation (training steps reuse the buffers)
template <typename V> int ensure(DevBuf<V>& d, size_t n) {
  if (d.n >= n && d.p) return BSP_OK;
  return d.alloc(std::max<size_t>(n, 1));
}

template <typename T> struct Model : ModelBase {
  bsp_learned_s* M;
  DevBuf<T> p, g, m, v, part;
  int64_t step = 0;
  bool dec_zero = true;  // parameters start at zero
  // per-matrix cache
  GraphBuf G;
  const bsp_matrix_s* cachedA = nullptr;
  int64_t cached_nnzb = -1;
  DevBuf<T> s, x, a, e, hs, msgs, ms, us;   // hs: (L+1) n H; msgs: L E H; ms, us: L n H
  DevBuf<T> dh, dh2, dm, gdr, gdc, de, gmh, gdF;
  DevBuf<double> dF, lz, lw, llam, ly, lu, le, lsc;
  std::unique_ptr<bsp_precond_s> work;   // learned LU of the cached matrix (ILU0 structure)

  explicit Model(bsp_learned_s* mm) : M(mm) {}

  const T* W(int slot) const { return p.get() + M->slots[slot].off; }
  const T* B(int slot) const {
    const ParamSlot& sl = M->slots[slot];
    return p.get() + sl.off + (int64_t)sl.nout * sl.nin;
  }
  T* Gp(int slot) { return g.get() + M->slots[slot].off; }

  int init() {
    const int64_t np = M->n_params;
    for (DevBuf<T>* b : {&p, &g, &m, &v}) {
      BSP_TRY(b->alloc(np));
      BSP_CUDA_TRY(cudaMemset(b->get(), 0, np * sizeof(T)));
    }
    BSP_TRY(part.alloc((size_t)kGradBlocks * (kB2 * 3 * H + kB2)));
    return BSP_OK;
  }

  int prepare(const bsp_matrix_s* A) {
    if (cachedA == A && G.A == A && G.n == A->n_rows && cached_nnzb == A->nnzb) return BSP_OK;
    BSP_TRY(build_graph(A, G));
    const int n = G.n, E = std::max(G.E, 1);
    BSP_TRY(s.alloc(n));
    BSP_TRY(x.alloc((size_t)n * (kB2 + 1)));
    BSP_TRY(a.alloc((size_t)E * kB2));
    BSP_TRY(e.alloc((size_t)E * H));
    BSP_TRY(hs.alloc((size_t)(kLayers + 1) * n * H));
    BSP_TRY(msgs.alloc((size_t)kLayers * E * H));
    BSP_TRY(ms.alloc((size_t)kLayers * n * H));
    BSP_TRY(us.alloc((size_t)kLayers * n * H));
    BSP_TRY(dF.alloc((size_t)A->nnzb * kB2));
    cachedA = A;
    cached_nnzb = A->nnzb;
    return BSP_OK;
  }

  // forward; writes dF (A order, FP64) into out (or the internal buffer)
  int run_forward(bsp_handle_s* h, const bsp_matrix_s* A, double* out) {
    BSP_TRY(prepare(A));
    const Graph gr = G.view();
    const int n = G.n, E = G.E, Es = std::max(E, 1);
    const int rg = (int)std::min<int64_t>(ceil_div((int64_t)std::max(n, E) * 32, 256), (int64_t)h->num_sms * 16);
    bsp::count_launch(), k_node_features<T><<<rg, 256, 0, h->stream>>>(gr, A->vals.get(), s.get(), x.get());
    if (E > 0) bsp::count_launch(), k_edge_features<T><<<rg, 256, 0, h->stream>>>(gr, A->vals.get(), s.get(), a.get());
    T* h0 = hs.get();
    BSP_TRY((run_dense<T, kB2 + 1, H>(h, n, W(0), B(0), RowIn<T, kB2 + 1>{x.get()}, ReluOut<T>{h0})));
    BSP_TRY((run_dense<T, kB2, H>(h, E, W(1), B(1), RowIn<T, kB2>{a.get()}, ReluOut<T>{e.get()})));
    for (int l = 0; l < kLayers; ++l) {
      T* hl = hs.get() + (size_t)l * n * H;
      T* hn = hs.get() + (size_t)(l + 1) * n * H;
      T* msg = msgs.get() + (size_t)l * Es * H;
      T* ml = ms.get() + (size_t)l * n * H;
      T* ul = us.get() + (size_t)l * n * H;
      BSP_TRY((run_dense<T, 2 * H, H>(h, E, W(2 + 2 * l), B(2 + 2 * l), MsgIn<T>{hl, e.get(), G.e_col.get()},
                                      ReluOut<T>{msg})));
      BSP_TRY((run_dense<T, 2 * H, H>(h, n, W(3 + 2 * l), B(3 + 2 * l), UpdIn<T>{hl, msg, G.er_ptr.get(), ml},
                                      ResidOut<T>{hl, ul, hn})));
    }
    const T* hL = hs.get() + (size_t)kLayers * n * H;
    const int so = 2 + 2 * kLayers;
    double* dst = out ? out : dF.get();
    const int llt = M->form == BSP_LEARNED_LLT;
    if (llt) BSP_CUDA_TRY(cudaMemsetAsync(dst, 0, (size_t)A->nnzb * kB2 * sizeof(double), h->stream));
    BSP_TRY((run_dense<T, 3 * H, kB2>(h, E, W(so), B(so), DecIn<T>{hL, e.get(), G.e_row.get(), G.e_col.get()},
                                      DecEdgeOut<T>{s.get(), G.e_row.get(), G.e_col.get(), G.e_blk.get(), dst,
                                                    llt})));
    BSP_TRY((run_dense<T, H, kB2>(h, n, W(so + 1), B(so + 1), RowIn<T, H>{hL},
                                  DecDiagOut<T>{s.get(), G.diag_pos.get(), dst, llt})));
    return BSP_OK;
  }

  int forward(bsp_handle_s* h, const bsp_matrix_s* A, double* out) override { return run_forward(h, A, out); }

  int loss_grad(bsp_handle_s* h, const bsp_matrix_s* A, const bsp_precond_s* ilu, int K, const double* probes,
                double* loss_out) override {
    BSP_TRY(run_forward(h, A, nullptr));
    const int n = G.n, E = G.E, Es = std::max(E, 1), bs = 8;
    const int64_t N = (int64_t)n * bs;
    const int llt = M->form == BSP_LEARNED_LLT;
    const int wkind = llt ? BSP_PC_LEARNED_LLT : BSP_PC_LEARNED_LU;
    if (!work || work->A != A || work->n != n || work->f_nnzb != ilu->f_nnzb || work->kind != wkind) {
      work = std::make_unique<bsp_precond_s>();
      work->h = h;
      work->device = h->device;
      work->A = const_cast<bsp_matrix_s*>(A);
      work->kind = wkind;
      work->n = n;
      work->bs = bs;
      work->precision = BSP_PREC_F64;
      BSP_TRY(precond_learned_init(work.get()));
    }
    work->relax = M->relax;
    BSP_TRY(precond_learned_refresh(work.get(), ilu, dF.get()));
    for (DevBuf<double>* b : {&lz, &lw, &llam, &ly}) BSP_TRY(ensure(*b, (size_t)N * K));
    BSP_TRY(ensure(lu, (size_t)N));
    BSP_TRY(ensure(le, (size_t)N));
    BSP_TRY(ensure(lsc, (size_t)K));
    BSP_TRY(ensure(gdF, (size_t)A->nnzb * kB2));
    for (DevBuf<T>* b : {&dh, &dh2, &dm}) BSP_TRY(ensure(*b, (size_t)n * H));
    for (DevBuf<T>* b : {&gdr, &gdc, &de, &gmh}) BSP_TRY(ensure(*b, (size_t)Es * H));
    const int eg = grid_for(h, N, 256);
    bsp_matrix_s* Am = const_cast<bsp_matrix_s*>(A);
    for (int k = 0; k < K; ++k) {
      const double* q = probes + (int64_t)k * N;
      double* z = lz.get() + (int64_t)k * N;
      BSP_TRY(bsmv_launch(Am, 1, 0, BSP_F64, 1.0, q, 0.0, nullptr, lu.get(), h->stream));
      BSP_TRY(precond_apply(work.get(), BSP_PREC_F64, lu.get(), z));
      bsp::count_launch(), k_diff<<<eg, 256, 0, h->stream>>>(N, z, q, le.get());
      BSP_TRY(bsp_dot_dev(h, N, le.get(), le.get(), lsc.get() + k));
      bsp::count_launch(), k_scale<<<eg, 256, 0, h->stream>>>(N, 2.0 / K, le.get());
      if (llt) {
        // w = M^-1 g (M = L L^T is symmetric); y = L^T z, u = L^T w (u in llam)
        double* wk = lw.get() + (int64_t)k * N;
        BSP_TRY(precond_apply(work.get(), BSP_PREC_F64, le.get(), wk));
        bsp::count_launch(), k_lower_t_prod<<<eg, 256, 0, h->stream>>>(
            n, bs, work->t_ptr.get(), work->t_row.get(), work->t_blk.get(), work->f_diag.get(), work->f_vals.get(), z,
            ly.get() + (int64_t)k * N);
        bsp::count_launch(), k_lower_t_prod<<<eg, 256, 0, h->stream>>>(
            n, bs, work->t_ptr.get(), work->t_row.get(), work->t_blk.get(), work->f_diag.get(), work->f_vals.get(), wk,
            llam.get() + (int64_t)k * N);
      } else {
        BSP_TRY(precond_apply_transposed(work.get(), le.get(), lw.get() + (int64_t)k * N, llam.get() + (int64_t)k * N));
        bsp::count_launch(), k_upper_prod<<<eg, 256, 0, h->stream>>>(n, bs, work->f_ptr.get(), work->f_col.get(),
                                                                     work->f_diag.get(), work->f_vals.get(), z,
                                                                     ly.get() + (int64_t)k * N);
      }
    }
    const int ng = (int)std::min<int64_t>(ceil_div((int64_t)n * 32, 256), (int64_t)h->num_sms * 16);
    if (llt) {
      // upper blocks of A are not in L: their gradient is zero
      BSP_CUDA_TRY(cudaMemsetAsync(gdF.get(), 0, (size_t)A->nnzb * kB2 * sizeof(T), h->stream));
      bsp::count_launch(), k_factor_grad_llt<T><<<ng, 256, 0, h->stream>>>(
          n, bs, K, N, work->f_ptr.get(), work->f_col.get(), work->f_diag.get(), work->d_perm.get(), lw.get(),
          ly.get(), lz.get(), llam.get(), gdF.get());
    } else {
      bsp::count_launch(), k_factor_grad<T><<<ng, 256, 0, h->stream>>>(n, bs, K, N, work->f_ptr.get(), work->f_col.get(),
                                                                      work->f_diag.get(), work->d_perm.get(), llam.get(),
                                                                      ly.get(), lw.get(), lz.get(), gdF.get());
    }
    BSP_CUDA_TRY(cudaPeekAtLastError());
    const Graph gr = G.view();
    // network backward: decoders
    const T* hL = hs.get() + (size_t)kLayers * n * H;
    const int so = 2 + 2 * kLayers;
    GEdgeDec<T> ge{s.get(), G.e_row.get(), G.e_col.get(), G.e_blk.get(), gdF.get(), llt};
    GDiagDec<T> gd{s.get(), G.diag_pos.get(), gdF.get(), llt};
    if (E > 0) {
      BSP_TRY((run_wgrad<T, 3 * H, kB2>(h, E, ge, DecIn<T>{hL, e.get(), G.e_row.get(), G.e_col.get()}, part.get(),
                                        Gp(so))));
      BSP_TRY((run_dense_t<T, 3 * H, kB2>(h, E, W(so), ge, SplitDecOut<T>{gdr.get(), gdc.get(), de.get()})));
    } else {
      BSP_CUDA_TRY(cudaMemsetAsync(Gp(so), 0, (size_t)(kB2 * 3 * H + kB2) * sizeof(T), h->stream));
    }
    BSP_TRY((run_wgrad<T, H, kB2>(h, n, gd, RowIn<T, H>{hL}, part.get(), Gp(so + 1))));
    BSP_TRY((run_dense_t<T, H, kB2>(h, n, W(so + 1), gd, DiagDhOut<T>{gr, gdr.get(), gdc.get(), dh.get()})));
    // message-passing layers, last first
    T* dcur = dh.get();
    T* dnext = dh2.get();
    for (int l = kLayers - 1; l >= 0; --l) {
      T* hl = hs.get() + (size_t)l * n * H;
      T* msg = msgs.get() + (size_t)l * Es * H;
      T* ml = ms.get() + (size_t)l * n * H;
      T* ul = us.get() + (size_t)l * n * H;
      GMask<T> gu{dcur, ul};
      BSP_TRY((run_wgrad<T, 2 * H, H>(h, n, gu, UpdInStored<T>{hl, ml}, part.get(), Gp(3 + 2 * l))));
      BSP_TRY((run_dense_t<T, 2 * H, H>(h, n, W(3 + 2 * l), gu, UpdBwdOut<T>{dcur, dnext, dm.get()})));
      if (E > 0) {
        GMaskRow<T> gm{dm.get(), msg, G.e_row.get()};
        BSP_TRY((run_wgrad<T, 2 * H, H>(h, E, gm, MsgIn<T>{hl, e.get(), G.e_col.get()}, part.get(), Gp(2 + 2 * l))));
        BSP_TRY((run_dense_t<T, 2 * H, H>(h, E, W(2 + 2 * l), gm, MsgBwdOut<T>{gmh.get(), de.get()})));
        bsp::count_launch(), k_gather_cols<T><<<ng, 256, 0, h->stream>>>(gr, gmh.get(), dnext);
      } else {
        BSP_CUDA_TRY(cudaMemsetAsync(Gp(2 + 2 * l), 0, (size_t)(H * 2 * H + H) * sizeof(T), h->stream));
      }
      std::swap(dcur, dnext);
    }
    if (E > 0)
      BSP_TRY((run_wgrad<T, kB2, H>(h, E, GMask<T>{de.get(), e.get()}, RowIn<T, kB2>{a.get()}, part.get(), Gp(1))));
    else
      BSP_CUDA_TRY(cudaMemsetAsync(Gp(1), 0, (size_t)(H * kB2 + H) * sizeof(T), h->stream));
    BSP_TRY((run_wgrad<T, kB2 + 1, H>(h, n, GMask<T>{dcur, hs.get()}, RowIn<T, kB2 + 1>{x.get()}, part.get(), Gp(0))));
    std::vector<double> lk(K);
    BSP_CUDA_TRY(cudaMemcpyAsync(lk.data(), lsc.get(), K * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    BSP_CUDA_TRY(cudaStreamSynchronize(h->stream));
    double L = 0.0;
    for (int k = 0; k < K; ++k) L += lk[k];
    *loss_out = L / K;
    BSP_TRY(precond_check_status(work.get()));
    return BSP_OK;
  }

  int adam(bsp_handle_s* h, double lr, double b1, double b2, double eps) override {
    ++step;
    dec_zero = false;
    const double c1 = 1.0 - std::pow(b1, (double)step), c2 = 1.0 - std::pow(b2, (double)step);
    bsp::count_launch(), k_adam<T><<<grid_for(h, M->n_params, 256), 256, 0, h->stream>>>(
        M->n_params, p.get(), g.get(), m.get(), v.get(), (T)lr, (T)b1, (T)b2, (T)eps, (T)c1, (T)c2);
    BSP_CUDA_TRY(cudaPeekAtLastError());
    return BSP_OK;
  }

  int get(double* out, int64_t cnt, int which) override {
    if (cnt < M->n_params) return BSP_INVALID;
    std::vector<T> tmp(M->n_params);
    BSP_CUDA_TRY(cudaMemcpy(tmp.data(), which ? g.get() : p.get(), M->n_params * sizeof(T), cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < M->n_params; ++i) out[i] = (double)tmp[i];
    return BSP_OK;
  }
  int set(const double* in, int64_t cnt) override {
    if (cnt != M->n_params) return BSP_INVALID;
    std::vector<T> tmp(in, in + cnt);
    // the decoders (Wo, bo, Wd, bd) are the last slots
    dec_zero = std::all_of(tmp.begin() + M->slots[2 + 2 * kLayers].off, tmp.end(), [](T x) { return x == T(0); });
    BSP_CUDA_TRY(cudaMemcpy(p.get(), tmp.data(), cnt * sizeof(T), cudaMemcpyHostToDevice));
    BSP_CUDA_TRY(cudaMemset(m.get(), 0, cnt * sizeof(T)));
    BSP_CUDA_TRY(cudaMemset(v.get(), 0, cnt * sizeof(T)));
    step = 0;
    return BSP_OK;
  }
  bool decoders_zero() const override { return dec_zero; }
};

}  // namespace

// ================================================================= C ABI
extern "C" {

int bsp_learned_create(bsp_handle_t h, int bs, int dtype, bsp_learned_t* out) {
  if (!h || !out) return BSP_INVALID;
  *out = nullptr;
  if (bs != 8 || (dtype != BSP_F32 && dtype != BSP_F64)) {
    record_error("the learned preconditioner supports 8x8 blocks and FP32 or FP64 arithmetic");
    return BSP_INVALID;
  }
  BSP_CUDA_TRY(cudaSetDevice(h->device));
  auto M = std::make_unique<bsp_learned_s>();
  M->h = h;
  M->device = h->device;
  M->bs = bs;
  M->dtype = dtype;
  M->slots = layout(M->n_params);
  if (dtype == BSP_F32) {
    auto m = std::make_unique<Model<float>>(M.get());
    BSP_TRY(m->init());
    M->impl = std::move(m);
  } else {
    auto m = std::make_unique<Model<double>>(M.get());
    BSP_TRY(m->init());
    M->impl = std::move(m);
  }
  *out = M.release();
  return BSP_OK;
}

int bsp_learned_set_form(bsp_learned_t M, int form) {
  if (!M || (form != BSP_LEARNED_LU && form != BSP_LEARNED_LLT)) return BSP_INVALID;
  M->form = form;
  return BSP_OK;
}

int bsp_learned_destroy(bsp_learned_t M) {
  if (!M) return BSP_OK;
  cudaSetDevice(M->device);
  delete M;
  return BSP_OK;
}

int bsp_learned_set_relax(bsp_learned_t M, double relax) {
  if (!M || !(relax > -1.0 && relax < 4.0)) return BSP_INVALID;
  M->relax = relax;
  return BSP_OK;
}

int bsp_learned_get_relax(bsp_learned_t M, double* relax) {
  if (!M || !relax) return BSP_INVALID;
  *relax = M->relax;
  return BSP_OK;
}

int bsp_learned_param_count(bsp_learned_t M, int64_t* count) {
  if (!M || !count) return BSP_INVALID;
  *count = M->n_params;
  return BSP_OK;
}

int bsp_learned_set_params(bsp_learned_t M, const double* params, int64_t count) {
  if (!M || !params) return BSP_INVALID;
  cudaSetDevice(M->device);
  return M->impl->set(params, count);
}

int bsp_learned_get_params(bsp_learned_t M, double* params, int64_t count) {
  if (!M || !params) return BSP_INVALID;
  cudaSetDevice(M->device);
  return M->impl->get(params, count, 0);
}

int bsp_learned_get_grads(bsp_learned_t M, double* grads, int64_t count) {
  if (!M || !grads) return BSP_INVALID;
  cudaSetDevice(M->device);
  return M->impl->get(grads, count, 1);
}

int bsp_learned_forward(bsp_handle_t h, bsp_learned_t M, bsp_matrix_t A, double* dF) {
  if (!h || !M || !A || !dF || A->bs != M->bs || A->n_rows != A->n_cols) return BSP_INVALID;
  BSP_CUDA_TRY(cudaSetDevice(h->device));
  BSP_TRY(M->impl->forward(h, A, dF));
  BSP_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return BSP_OK;
}

int bsp_learned_ilu_factors(bsp_handle_t h, bsp_precond_t ilu, double* F0) {
  if (!h || !ilu || !F0 || (ilu->kind != BSP_PC_ILU0 && ilu->kind != BSP_PC_ICHOL0)) return BSP_INVALID;
  BSP_CUDA_TRY(cudaSetDevice(h->device));
  const int b2 = ilu->bs * ilu->bs;
  // IChol0 covers A's lower blocks only: the others are zero
  BSP_CUDA_TRY(cudaMemsetAsync(F0, 0, (size_t)ilu->A->nnzb * b2 * sizeof(double), h->stream));
  bsp::count_launch(), k_scatter_f0<<<grid_for(h, ilu->f_nnzb * b2, 256), 256, 0, h->stream>>>(
      ilu->f_nnzb, b2, ilu->d_perm.get(), ilu->f_vals.get(), F0);
  BSP_CUDA_TRY(cudaPeekAtLastError());
  BSP_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return BSP_OK;
}

int bsp_learned_loss_grad(bsp_handle_t h, bsp_learned_t M, bsp_matrix_t A, bsp_precond_t ilu, int n_probes,
                          const double* probes, double* loss) {
  if (!h || !M || !A || !ilu || !probes || !loss || n_probes < 1 || A->bs != M->bs || ilu->A != A ||
      ilu->kind != (M->form == BSP_LEARNED_LLT ? BSP_PC_ICHOL0 : BSP_PC_ILU0))
    return BSP_INVALID;
  BSP_CUDA_TRY(cudaSetDevice(h->device));
  return M->impl->loss_grad(h, A, ilu, n_probes, probes, loss);
}

int bsp_learned_adam_step(bsp_handle_t h, bsp_learned_t M, double lr, double beta1, double beta2, double eps) {
  if (!h || !M) return BSP_INVALID;
  BSP_CUDA_TRY(cudaSetDevice(h->device));
  return M->impl->adam(h, lr, beta1, beta2, eps);
}

int bsp_learned_probes(bsp_handle_t h, bsp_matrix_t A, bsp_precond_t pc, const double* b, int K, double* probes) {
  if (!h || !A || !b || !probes || K < 1) return BSP_INVALID;
  BSP_CUDA_TRY(cudaSetDevice(h->device));
  const int64_t N = (int64_t)A->n_rows * A->bs;
  DevBuf<double> v, sc;
  BSP_TRY(v.alloc(N));
  BSP_TRY(sc.alloc(2));
  const int g = grid_for(h, N, 256);
  // q_0 = M^-1 b / ||.||; q_{j+1} = orthonormalised M^-1 A q_j (modified Gram-Schmidt)
  BSP_CUDA_TRY(cudaMemcpyAsync(v.get(), b, N * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  if (pc) BSP_TRY(precond_apply(pc, BSP_PREC_F64, v.get(), v.get()));
  for (int j = 0; j < K; ++j) {
    if (j > 0) {
      BSP_TRY(bsmv_launch(A, 1, 0, BSP_F64, 1.0, probes + (int64_t)(j - 1) * N, 0.0, nullptr, v.get(), h->stream));
      if (pc) BSP_TRY(precond_apply(pc, BSP_PREC_F64, v.get(), v.get()));
      for (int i = 0; i < j; ++i) {
        BSP_TRY(bsp_dot_dev(h, N, probes + (int64_t)i * N, v.get(), sc.get()));
        bsp::count_launch(), k_sub_proj<<<g, 256, 0, h->stream>>>(N, sc.get(), probes + (int64_t)i * N, v.get());
      }
    }
    BSP_TRY(bsp_dot_dev(h, N, v.get(), v.get(), sc.get() + 1));
    bsp::count_launch(), k_normalize<<<g, 256, 0, h->stream>>>(N, v.get(), sc.get() + 1, probes + (int64_t)j * N);
  }
  BSP_CUDA_TRY(cudaPeekAtLastError());
  BSP_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return BSP_OK;
}

int bsp_learned_smooth(bsp_handle_t h, bsp_matrix_t A, bsp_precond_t pc, int K, int steps, double* vecs) {
  if (!h || !A || !pc || !vecs || K < 1 || steps < 0) return BSP_INVALID;
  BSP_CUDA_TRY(cudaSetDevice(h->device));
  const int64_t N = (int64_t)A->n_rows * A->bs;
  DevBuf<double> t, sc;
  BSP_TRY(t.alloc(N));
  BSP_TRY(sc.alloc(2));
  const int g = grid_for(h, N, 256);
  for (int k = 0; k < K; ++k) {
    double* v = vecs + (int64_t)k * N;
    // e <- e - M^-1 A e: the error of the preconditioned stationary iteration
    for (int s = 0; s < steps; ++s) {
      BSP_TRY(bsmv_launch(A, 1, 0, BSP_F64, 1.0, v, 0.0, nullptr, t.get(), h->stream));
      BSP_TRY(precond_apply(pc, BSP_PREC_F64, t.get(), t.get()));
      bsp::count_launch(), k_sub_one<<<g, 256, 0, h->stream>>>(N, t.get(), v);
    }
    for (int i = 0; i < k; ++i) {
      BSP_TRY(bsp_dot_dev(h, N, vecs + (int64_t)i * N, v, sc.get()));
      bsp::count_launch(), k_sub_proj<<<g, 256, 0, h->stream>>>(N, sc.get(), vecs + (int64_t)i * N, v);
    }
    BSP_TRY(bsp_dot_dev(h, N, v, v, sc.get() + 1));
    bsp::count_launch(), k_normalize<<<g, 256, 0, h->stream>>>(N, v, sc.get() + 1, v);
  }
  BSP_CUDA_TRY(cudaPeekAtLastError());
  BSP_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return BSP_OK;
}

int bsp_learned_precond(bsp_handle_t h, bsp_learned_t M, bsp_matrix_t A, int precision, bsp_precond_t* out) {
  if (!h || !M || !A || !out || A->bs != M->bs || A->n_rows != A->n_cols || A->cbs) return BSP_INVALID;
  *out = nullptr;
  BSP_CUDA_TRY(cudaSetDevice(h->device));
  // zero decoders give dF = 0 exactly: the factors are the (relaxed) baseline's
  DevBuf<double> dF;
  if (!M->impl->decoders_zero()) {
    BSP_TRY(dF.alloc((size_t)A->nnzb * A->bs * A->bs));
    BSP_TRY(M->impl->forward(h, A, dF.get()));
  }
  auto pc = std::make_unique<bsp_precond_s>();
  pc->h = h;
  pc->device = h->device;
  pc->A = A;
  pc->kind = M->form == BSP_LEARNED_LLT ? BSP_PC_LEARNED_LLT : BSP_PC_LEARNED_LU;
  pc->n = A->n_rows;
  pc->bs = A->bs;
  pc->precision = precision;
  pc->relax = M->relax;
  if (precision != BSP_PREC_F64)
    BSP_TRY(bsp_matrix_make_lowp(A, precision == BSP_PREC_F32 ? BSP_F32 : BSP_BF16));
  BSP_TRY(precond_build_learned(pc.get(), dF.get()));
  BSP_CUDA_TRY(cudaStreamSynchronize(h->stream));
  *out = pc.release();
  return BSP_OK;
}

}  // extern "C"
