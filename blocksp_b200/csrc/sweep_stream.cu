// sweep_stream.cu — the streamed block triangular sweep on sm_100a.
//
// Reference: blocksp_preconditioners.hpp:294-349 (ILU0::invmul: unit-L
// forward substitution, then backward substitution with D_Inv[i] = U_ii^-1)
// and :432-489 (IChol0::invmul: L forward with L_ii^-1, then L^T backward
// through the column structure of L with L_ii^-T).  Natural order is kept:
// a row runs once every row it reads is final, and computes exactly the
// reference's row update.
//
// Execution (one persistent launch per sweep):
//   * a CTA claims a super-task (W chains: a tile of consecutive chains by
//     chains one plane apart, or W consecutive chains) with an atomic ticket,
//     in dependency-level order; warp w runs chain w row by row;
//   * a row of another super-task is read from global memory: the output
//     vector is pre-filled with a signalling-NaN sentinel and a row is
//     published by its values, so a consumer polls the words it needs
//     (bounded spin) until they differ from the sentinel;
//   * a row of another chain of the same CTA is read from that warp's output
//     rows in shared memory, which are published the same way (sentinel
//     until written), so neither side needs a memory fence;
//   * the chain's previous row is passed on in registers;
//   * every block of the row, its D block and its right-hand side are staged
//     DEPTH rows ahead into a per-warp shared-memory ring by per-lane cp.async
//     copies of the contiguous stream (each lane copies exactly the chunks it
//     reads later, so it only waits for its own copies); the values of the
//     row's external dependencies are copied into the ring at the same time,
//     so a dependency published by then costs no round trip when the row
//     starts (a copy that still holds the sentinel is polled in global
//     memory).
// Lane map: a block of BS x BS values of type VT is 32*P chunks of V values;
// lane l holds chunk q*32 + l (block row q*RPP + l/CPR, columns c0..c0+V-1,
// c0 = (l % CPR)*V), so a row's dot products end in a CPR-lane reduction.
// Accumulation is FP64 for every storage type (vectors are FP64).
#include <algorithm>
#include <map>
#include <numeric>
#include "sentinel.cuh"
#include "stage.cuh"
#include "sweep_stream.hpp"

namespace bsp {

// ------------------------------------------------------------------ lane map
template <int BS, typename VT> struct SMap {
  static constexpr int V0 = 16 / (int)sizeof(VT);
  static constexpr int VF = BS * BS / 32;
  static constexpr int V = VF < V0 ? VF : V0;  // values per lane chunk
  static_assert(V >= 1 && BS % V == 0, "block too small for a 32-lane map");
  static constexpr int CB = V * (int)sizeof(VT);  // 4, 8 or 16 bytes
  static constexpr int CPR = BS / V;
  static constexpr int CPB = BS * BS / V;
  static constexpr int P = CPB / 32;
  static constexpr int RPP = 32 / CPR;
  static constexpr int BB = BS * BS * (int)sizeof(VT);
  static_assert(CPB % 32 == 0 && 32 % CPR == 0, "unsupported block map");
};

template <int N> __device__ __forceinline__ void cp_async_n(void* dst, const void* src) {
  if constexpr (N == 16) cp_async16(dst, src);
  else cp_async_small<N>(dst, src);
}

// One lane chunk (V values of VT) from shared or global memory, as doubles.
template <typename VT, int V> struct ChunkOps;
template <> struct ChunkOps<double, 2> {
  __device__ static void get(const void* p, double (&a)[2]) {
    const double2 t = *reinterpret_cast<const double2*>(p);
    a[0] = t.x; a[1] = t.y;
  }
};
template <> struct ChunkOps<float, 2> {
  __device__ static void get(const void* p, double (&a)[2]) {
    const float2 t = *reinterpret_cast<const float2*>(p);
    a[0] = t.x; a[1] = t.y;
  }
};
template <> struct ChunkOps<float, 4> {
  __device__ static void get(const void* p, double (&a)[4]) {
    const float4 t = *reinterpret_cast<const float4*>(p);
    a[0] = t.x; a[1] = t.y; a[2] = t.z; a[3] = t.w;
  }
};
template <> struct ChunkOps<__nv_bfloat16, 2> {
  __device__ static void get(const void* p, double (&a)[2]) {
    const float2 f = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(p));
    a[0] = f.x; a[1] = f.y;
  }
};
template <> struct ChunkOps<__nv_bfloat16, 8> {
  __device__ static void get(const void* p, double (&a)[8]) {
    const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(p);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const float2 f = __bfloat1622float2(h[i]);
      a[2 * i] = f.x; a[2 * i + 1] = f.y;
    }
  }
};

template <typename VT> struct SSP {
  int n_super;
  const int* super_beg;
  const int4* chains;
  const int4* rec;
  const int* codes;
  const VT* vals;
  const VT* dvals;
  const double* rhs;
  double* x;
  int dir;
  unsigned spin_limit;
  unsigned* ticket;
  DevStatus* st;
};

template <int BS, typename VT, bool HAS_D, int W, int DEPTH> struct SSCfg {
  using M = SMap<BS, VT>;
  static constexpr int OFF_D = kStreamEmax * M::BB;
  static constexpr int OFF_R = OFF_D + (HAS_D ? M::BB : 0);
  static constexpr int OFF_X = OFF_R + BS * 8;               // + the row's right-hand side
  static constexpr int SB = OFF_X + kStreamEmax * BS * 8;    // + the staged rows' external x values
  static constexpr size_t RING = (size_t)W * DEPTH * SB;
  static constexpr size_t BUF = (size_t)W * kStreamCmax * BS * 8;   // output rows of each chain
  static constexpr size_t REC = (size_t)W * kStreamCmax * 16;       // row records of each chain
  static constexpr size_t EOF_ = (size_t)W * kStreamCmax * 4;       // entry offsets of each row
  static constexpr size_t kSmem = RING + BUF + REC + EOF_;
};

__device__ __forceinline__ bool failed(const DevStatus* st) {
  return *reinterpret_cast<const volatile int*>(&st->code) != 0;
}

template <int BS, typename VT, bool HAS_D, int W, int DEPTH>
__global__ void __launch_bounds__(W * 32) k_ssweep(const SSP<VT> p) {
  using M = SMap<BS, VT>;
  using C = SSCfg<BS, VT, HAS_D, W, DEPTH>;
  constexpr int V = M::V, P = M::P, CPR = M::CPR, RPP = M::RPP, BB = M::BB, CB = M::CB;
  extern __shared__ __align__(128) unsigned char ss_smem[];
  __shared__ int s_task;
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  const int c0 = (l % CPR) * V;
  unsigned char* ring = ss_smem + (size_t)w * DEPTH * C::SB;
  double* buf_all = reinterpret_cast<double*>(ss_smem + C::RING);
  double* buf = buf_all + (size_t)w * kStreamCmax * BS;
  int4* rw = reinterpret_cast<int4*>(ss_smem + C::RING + C::BUF) + w * kStreamCmax;
  int* eo = reinterpret_cast<int*>(ss_smem + C::RING + C::BUF + C::REC) + w * kStreamCmax;
  const unsigned limit = p.spin_limit;
  DevStatus* const st = p.st;
  double* const xg = p.x;

  while (true) {
    if (threadIdx.x == 0) s_task = (int)atomicAdd(p.ticket, 1u);
    // the chain's output rows in shared memory are published by their values,
    // like the global vector: the sentinel until the row is written
    for (int x = l; x < kStreamCmax * BS; x += 32)
      reinterpret_cast<unsigned long long*>(buf)[x] = kSentinel64;
    __syncthreads();
    const int t = s_task;
    if (t >= p.n_super) break;
    const int c = __ldg(p.super_beg + t) + w;
    if (c < __ldg(p.super_beg + t + 1)) {
      const int4 ch = __ldg(p.chains + c);
      const int row0 = ch.x, len = ch.y, q0 = ch.z, e0 = ch.w;
      // the chain's row records and entry offsets (exclusive scan of n_e)
      {
        int4 ra = make_int4(0, 0, 0, 0), rb = make_int4(0, 0, 0, 0);
        if (l < len) ra = __ldg(p.rec + q0 + l);
        if (l + 32 < len) rb = __ldg(p.rec + q0 + 32 + l);
        int ia = ra.w, ib = rb.w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int ta = __shfl_up_sync(0xffffffffu, ia, o);
          const int tb = __shfl_up_sync(0xffffffffu, ib, o);
          if (l >= o) { ia += ta; ib += tb; }
        }
        const int tot_a = __shfl_sync(0xffffffffu, ia, 31);
        rw[l] = ra;
        rw[32 + l] = rb;
        eo[l] = e0 + ia - ra.w;
        eo[32 + l] = e0 + tot_a + ib - rb.w;
      }
      __syncwarp();
      // stage row s of the chain into ring slot s % DEPTH (one commit group)
      auto issue = [&](int s) {
        if (s < len) {
          const int4 rr = rw[s];
          const int ne = rr.w < kStreamEmax ? rr.w : kStreamEmax;
          unsigned char* dst = ring + (s % DEPTH) * C::SB;
          const unsigned char* vs = reinterpret_cast<const unsigned char*>(p.vals) + (int64_t)eo[s] * BB;
#pragma unroll
          for (int u = 0; u < kStreamEmax; ++u)
            if (u < ne) {
#pragma unroll
              for (int q = 0; q < P; ++q) cp_async_n<CB>(dst + u * BB + (q * 32 + l) * CB, vs + u * BB + (q * 32 + l) * CB);
            }
          if constexpr (HAS_D) {
            const unsigned char* ds = reinterpret_cast<const unsigned char*>(p.dvals) + (int64_t)(q0 + s) * BB;
#pragma unroll
            for (int q = 0; q < P; ++q) cp_async_n<CB>(dst + C::OFF_D + (q * 32 + l) * CB, ds + (q * 32 + l) * CB);
          }
          const int r = row0 + s * p.dir;
          if (l < BS / 2) cp_async16(dst + C::OFF_R + l * 16, p.rhs + (int64_t)r * BS + 2 * l);
          // the external rows' values as they are now: published ones are
          // final, the others still hold the sentinel and are polled later
          const int code[kStreamEmax] = {rr.x, rr.y, rr.z};
#pragma unroll
          for (int u = 0; u < kStreamEmax; ++u)
            if (u < ne && code[u] >= 0 && l < BS / 2)
              cp_async16(dst + C::OFF_X + u * BS * 8 + l * 16, xg + (int64_t)code[u] * BS + 2 * l);
        }
        cp_async_commit();
      };
#pragma unroll
      for (int s = 0; s < DEPTH; ++s) issue(s);

      double prev[V];
#pragma unroll
      for (int v = 0; v < V; ++v) prev[v] = 0.0;
      // the next row's external values, loaded one row ahead: a dependency
      // published after the ring copy was made but before this load is
      // still found without a round trip on the row's path
      double nx[kStreamEmax][V];
      auto load_next = [&](int s2) {
        if (s2 < len) {
          const int4 r2 = rw[s2];
          const int c2[kStreamEmax] = {r2.x, r2.y, r2.z};
#pragma unroll
          for (int u = 0; u < kStreamEmax; ++u)
            if (u < r2.w && c2[u] >= 0) ld_vec_cg<V>(xg + (int64_t)c2[u] * BS + c0, nx[u]);
        }
      };
      load_next(0);
      auto poll = [&](int j, double (&xv)[V], int who) {
        bool pend = false;
#pragma unroll
        for (int v = 0; v < V; ++v) pend |= is_sentinel(xv[v]);
        unsigned spins = 0;
        while (pend) {
          if (++spins > limit) {
            set_status(st, BSP_TIMEOUT, who);
            break;
          }
          if ((spins & 255u) == 0u && failed(st)) break;
          poll_pause(spins);
#pragma unroll
          for (int v = 0; v < V; ++v) xv[v] = ld_poll(xg + (int64_t)j * BS + c0 + v);
          pend = false;
#pragma unroll
          for (int v = 0; v < V; ++v) pend |= is_sentinel(xv[v]);
        }
      };
      // a row of another chain of this CTA: its words in that warp's output
      // rows, read until they are no longer the sentinel (no fence needed)
      auto local = [&](int slot, double (&xv)[V], int who) {
        const int ww = slot / kStreamCmax, ss = slot - ww * kStreamCmax;
        const volatile double* src = buf_all + ((size_t)ww * kStreamCmax + ss) * BS + c0;
        bool pend = false;
#pragma unroll
        for (int v = 0; v < V; ++v) {
          xv[v] = src[v];
          pend |= is_sentinel(xv[v]);
        }
        unsigned spins = 0;
        while (pend) {
          if (++spins > limit) {
            set_status(st, BSP_TIMEOUT, who);
            break;
          }
          if ((spins & 255u) == 0u && failed(st)) break;
          if (spins >= kSpinFree) __nanosleep(32);
          pend = false;
#pragma unroll
          for (int v = 0; v < V; ++v) {
            xv[v] = src[v];
            pend |= is_sentinel(xv[v]);
          }
        }
      };
      auto fma_chunks = [&](const unsigned char* blk, const double (&xv)[V], double (&acc)[P]) {
#pragma unroll
        for (int q = 0; q < P; ++q) {
          double a[V];
          ChunkOps<VT, V>::get(blk + (q * 32 + l) * CB, a);
#pragma unroll
          for (int v = 0; v < V; ++v) acc[q] = fma(a[v], xv[v], acc[q]);
        }
      };

      for (int s = 0; s < len; ++s) {
        const int r = row0 + s * p.dir;
        const int4 rr = rw[s];
        const int ne = rr.w;
        cp_async_wait<DEPTH - 1>();
        __syncwarp();  // the prefetched x values were copied by lanes 0..BS/2-1
        const unsigned char* sl = ring + (s % DEPTH) * C::SB;
        // the row's staged blocks and its D rhs part do not depend on the
        // sweep: read from shared memory before any dependency is awaited,
        // so the waits and these reads overlap
        double blk[kStreamEmax][P][V];
#pragma unroll
        for (int u = 0; u < kStreamEmax; ++u)
          if (u < ne) {
#pragma unroll
            for (int q = 0; q < P; ++q) ChunkOps<VT, V>::get(sl + u * BB + (q * 32 + l) * CB, blk[u][q]);
          }
        const double* rh = reinterpret_cast<const double*>(sl + C::OFF_R);
        double base[P];  // D_r rhs_r partial of this lane (with D), or rhs_r
#pragma unroll
        for (int q = 0; q < P; ++q) {
          if constexpr (HAS_D) {
            double a[V];
            ChunkOps<VT, V>::get(sl + C::OFF_D + (q * 32 + l) * CB, a);
            double o = 0.0;
#pragma unroll
            for (int v = 0; v < V; ++v) o = fma(a[v], rh[c0 + v], o);
            base[q] = o;
          } else {
            base[q] = rh[q * RPP + l / CPR];
          }
        }
        double acc[P];
#pragma unroll
        for (int q = 0; q < P; ++q) acc[q] = 0.0;
        const int code[kStreamEmax] = {rr.x, rr.y, rr.z};
        double xv[kStreamEmax][V];
        // external rows: the values copied with the row's blocks, else the
        // ones loaded a row ahead; only a row published after both is polled
#pragma unroll
        for (int u = 0; u < kStreamEmax; ++u)
          if (u < ne && code[u] >= 0) {
            const double* px = reinterpret_cast<const double*>(sl + C::OFF_X + u * BS * 8) + c0;
            bool ring_ok = true;
#pragma unroll
            for (int v = 0; v < V; ++v) {
              xv[u][v] = px[v];
              ring_ok &= !is_sentinel(xv[u][v]);
            }
            if (!ring_ok) {
#pragma unroll
              for (int v = 0; v < V; ++v) xv[u][v] = nx[u][v];
            }
          }
        load_next(s + 1);
#pragma unroll
        for (int u = 0; u < kStreamEmax; ++u) {
          if (u < ne) {
            if (code[u] >= 0) poll(code[u], xv[u], r);
            else if (code[u] == -1) {
#pragma unroll
              for (int v = 0; v < V; ++v) xv[u][v] = prev[v];
            } else {
              local(-code[u] - 2, xv[u], r);
            }
#pragma unroll
            for (int q = 0; q < P; ++q)
#pragma unroll
              for (int v = 0; v < V; ++v) acc[q] = fma(blk[u][q][v], xv[u][v], acc[q]);
          }
        }
        // rows with more entries than are staged: codes and blocks from global memory
        for (int u = kStreamEmax; u < ne; ++u) {
          const int e = eo[s] + u;
          const int cd = __ldg(p.codes + e);
          double xe[V];
          if (cd >= 0) {
            ld_vec_cg<V>(xg + (int64_t)cd * BS + c0, xe);
            poll(cd, xe, r);
          } else if (cd == -1) {
#pragma unroll
            for (int v = 0; v < V; ++v) xe[v] = prev[v];
          } else {
            local(-cd - 2, xe, r);
          }
          fma_chunks(reinterpret_cast<const unsigned char*>(p.vals) + (int64_t)e * BB, xe, acc);
        }
        // x_r = rhs_r - sum (no D), or D_r rhs_r - sum with the blocks
        // premultiplied by D_r; the CPR lanes of each block row then reduce
        double xr[P];
#pragma unroll
        for (int q = 0; q < P; ++q) {
          if constexpr (HAS_D) xr[q] = row_reduce<CPR>(base[q] - acc[q], 0xffffffffu);
          else xr[q] = base[q] - row_reduce<CPR>(acc[q], 0xffffffffu);
        }
        // publish row r by its values: shared memory first (this CTA's next
        // chains poll it there), then global memory (other CTAs poll it)
        double* bro = buf + s * BS;
        if (l % CPR == 0) {
#pragma unroll
          for (int q = 0; q < P; ++q) bro[q * RPP + l / CPR] = xr[q];
        }
        __syncwarp();
        if (l % CPR == 0) {
#pragma unroll
          for (int q = 0; q < P; ++q) xg[(int64_t)r * BS + q * RPP + l / CPR] = xr[q];
        }
#pragma unroll
        for (int v = 0; v < V; ++v) prev[v] = bro[c0 + v];
        issue(s + DEPTH);
      }
      cp_async_wait<0>();
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------------ gathers
// dst[e] (VT, bs x bs, transposed when trans) = src[idx[e]] (FP64)
template <typename VT, typename IT>
__global__ void k_stream_gather(int64_t nblk, int bs, const IT* __restrict__ idx, const double* __restrict__ src,
                                int trans, VT* __restrict__ dst) {
  const int b2 = bs * bs;
  const int64_t total = nblk * b2;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = t / b2;
    const int k = (int)(t - e * b2);
    const int a = k / bs, c = k - a * bs;
    const double v = src[(int64_t)idx[e] * b2 + (trans ? c * bs + a : k)];
    if constexpr (std::is_same<VT, double>::value) dst[t] = v;
    else if constexpr (std::is_same<VT, float>::value) dst[t] = (float)v;
    else dst[t] = __float2bfloat16_rn((float)v);
  }
}

// dst[e] (VT) = D_r B_e in FP64, r the row of entry e: D = dinv[r] (transposed
// when trans_d), B_e = src[idx[e]] (transposed when trans).
template <typename VT>
__global__ void k_stream_gather_premul(int64_t nblk, int bs, const int64_t* __restrict__ idx,
                                       const int* __restrict__ ent_q, const int* __restrict__ q_row,
                                       const double* __restrict__ src, const double* __restrict__ dinv, int trans,
                                       int trans_d, VT* __restrict__ dst) {
  const int b2 = bs * bs;
  const int64_t total = nblk * b2;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = t / b2;
    const int k = (int)(t - e * b2);
    const int a = k / bs, c = k - a * bs;
    const double* D = dinv + (int64_t)q_row[ent_q[e]] * b2;
    const double* B = src + (int64_t)idx[e] * b2;
    double v = 0.0;
    for (int m = 0; m < bs; ++m)
      v = fma(trans_d ? D[m * bs + a] : D[a * bs + m], trans ? B[c * bs + m] : B[m * bs + c], v);
    if constexpr (std::is_same<VT, double>::value) dst[t] = v;
    else if constexpr (std::is_same<VT, float>::value) dst[t] = (float)v;
    else dst[t] = __float2bfloat16_rn((float)v);
  }
}

int grid_for(const bsp_handle_s* h, int64_t n, int threads);

// ------------------------------------------------------------------ host: build
bool stream_supported(int bs) { return bs == 8 || bs == 16; }

int stream_warps(int bs) { return bs >= 16 ? 4 : 16; }

template <typename T> static int upload_vec(DevBuf<T>& d, const std::vector<T>& v) {
  BSP_TRY(d.alloc(v.empty() ? 1 : v.size()));
  if (!v.empty()) BSP_CUDA_TRY(cudaMemcpy(d.get(), v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  return BSP_OK;
}

int stream_plan(int n, bool ascending, int warps, const SweepEntries& E, StreamPlan& S) {
  const int dir = ascending ? 1 : -1;
  S.n = n;
  S.W = warps;
  S.dir = dir;
  // chains in sweep order: row r continues the chain of r - dir when it
  // depends on that row and the chain is shorter than kStreamCmax
  std::vector<int> chain_of(n), pos(n), first, clen;
  for (int idx = 0; idx < n; ++idx) {
    const int r = ascending ? idx : n - 1 - idx;
    const int pr = r - dir;
    bool cont = false;
    if (idx > 0 && clen[chain_of[pr]] < kStreamCmax)
      for (int t = E.ptr[r]; t < E.ptr[r + 1]; ++t) cont |= (E.col[t] == pr);
    if (cont) {
      const int c = chain_of[pr];
      chain_of[r] = c;
      pos[r] = clen[c]++;
    } else {
      chain_of[r] = (int)first.size();
      pos[r] = 0;
      first.push_back(r);
      clen.push_back(1);
    }
  }
  const int nc = (int)first.size();
  // chain dependencies (distinct predecessor chains) and their strides
  std::vector<std::vector<int>> cdeps(nc);
  std::map<int, int> stride_count;
  for (int c = 0; c < nc; ++c) {
    auto& dc = cdeps[c];
    for (int k = 0; k < clen[c]; ++k) {
      const int r = first[c] + k * dir;
      for (int t = E.ptr[r]; t < E.ptr[r + 1]; ++t)
        if (chain_of[E.col[t]] != c) dc.push_back(chain_of[E.col[t]]);
    }
    std::sort(dc.begin(), dc.end());
    dc.erase(std::unique(dc.begin(), dc.end()), dc.end());
    for (int cj : dc)
      if (c - cj >= 2) stride_count[c - cj]++;
  }
  // super-tasks: tiles of wy consecutive chains by wz chains strided by d
  // (the chain's neighbour in the next plane of a grid), so that both
  // directions across the chains stay inside the CTA; warps in tile order
  std::vector<int> sup_of(nc), warp_of(nc), lvl;
  std::vector<std::vector<int>> members, succ;
  int nsup = 0;
  auto tile = [&](int d, int wy, int wz) {
    const int cols = (d + wy - 1) / wy;
    std::map<int64_t, int> ids;
    std::vector<int> key_warp(nc);
    for (int c = 0; c < nc; ++c) {
      const int a = c / (wz * d), rem = c % (wz * d), zi = rem / d, o = rem % d;
      const int64_t key = (int64_t)a * cols + o / wy;
      auto it = ids.find(key);
      if (it == ids.end()) it = ids.emplace(key, (int)ids.size()).first;
      sup_of[c] = it->second;
      key_warp[c] = zi * wy + o % wy;
    }
    nsup = (int)ids.size();
    members.assign(nsup, {});
    for (int c = 0; c < nc; ++c) members[sup_of[c]].push_back(c);
    for (auto& m : members) {
      std::sort(m.begin(), m.end(), [&](int x, int y) { return key_warp[x] < key_warp[y]; });
      for (int i = 0; i < (int)m.size(); ++i) warp_of[m[i]] = i;
    }
    // super-task graph and its longest-path levels (Kahn); false on a cycle
    succ.assign(nsup, {});
    std::vector<int> indeg(nsup, 0), queue;
    for (int c = 0; c < nc; ++c)
      for (int cj : cdeps[c])
        if (sup_of[cj] != sup_of[c]) succ[sup_of[cj]].push_back(sup_of[c]);
    for (auto& v : succ) {
      std::sort(v.begin(), v.end());
      v.erase(std::unique(v.begin(), v.end()), v.end());
      for (int b : v) indeg[b]++;
    }
    lvl.assign(nsup, 0);
    for (int a = 0; a < nsup; ++a)
      if (!indeg[a]) queue.push_back(a);
    for (size_t h = 0; h < queue.size(); ++h)
      for (int b : succ[queue[h]]) {
        lvl[b] = std::max(lvl[b], lvl[queue[h]] + 1);
        if (--indeg[b] == 0) queue.push_back(b);
      }
    return (int)queue.size() == nsup;
  };
  int dom = 0, dom_n = 0;
  for (auto& kv : stride_count)
    if (kv.second > dom_n) {
      dom = kv.first;
      dom_n = kv.second;
    }
  int wz = 1;
  while (wz * wz * 4 <= warps) wz *= 2;  // 16 -> 4 x 4, 8 -> 4 x 2, 4 -> 2 x 2
  const int wy = warps / wz;
  S.stride = 0;
  if (warps > 1 && wz > 1 && dom >= wy && dom_n * 2 >= nc && tile(dom, wy, wz)) {
    S.stride = dom;
  } else if (!tile(std::max(nc, 1), warps, 1)) {  // W consecutive chains
    record_error("streamed sweep: dependency graph is not triangular");
    return BSP_INVALID;
  }
  int maxl = 0;
  for (int v : lvl) maxl = std::max(maxl, v);
  S.n_levels = maxl + 1;
  std::vector<int> order(nsup);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return lvl[a] < lvl[b]; });
  // stream layout in ticket order
  std::vector<int> super_beg(nsup + 1, 0), codes, q_row(n), ent_q;
  std::vector<int4> chains, rec(n);
  std::vector<int64_t> src;
  codes.reserve(E.col.size());
  src.reserve(E.col.size());
  ent_q.reserve(E.col.size());
  chains.reserve(nc);
  int q = 0;
  std::vector<std::pair<int, int64_t>> ext, loc;
  std::pair<int, int64_t> inchain;
  for (int t = 0; t < nsup; ++t) {
    const int sp = order[t];
    super_beg[t] = (int)chains.size();
    for (int c : members[sp]) {
      chains.push_back(make_int4(first[c], clen[c], q, (int)codes.size()));
      for (int k = 0; k < clen[c]; ++k, ++q) {
        const int r = first[c] + k * dir;
        q_row[q] = r;
        ext.clear();
        loc.clear();
        bool has_in = false;
        for (int tt = E.ptr[r]; tt < E.ptr[r + 1]; ++tt) {
          const int j = E.col[tt], cj = chain_of[j];
          if (cj == c && pos[j] == k - 1) {
            has_in = true;
            inchain = {-1, E.blk[tt]};
          } else if (sup_of[cj] == sp) {
            loc.emplace_back(-2 - (warp_of[cj] * kStreamCmax + pos[j]), E.blk[tt]);
          } else {
            ext.emplace_back(j, E.blk[tt]);
          }
        }
        const int e_first = (int)codes.size();
        for (auto& e : ext) { codes.push_back(e.first); src.push_back(e.second); }
        for (auto& e : loc) { codes.push_back(e.first); src.push_back(e.second); }
        if (has_in) { codes.push_back(-1); src.push_back(inchain.second); }
        const int ne = (int)codes.size() - e_first;
        ent_q.insert(ent_q.end(), ne, q);
        int cc[3] = {0, 0, 0};
        for (int u = 0; u < std::min(ne, 3); ++u) cc[u] = codes[e_first + u];
        rec[q] = make_int4(cc[0], cc[1], cc[2], ne);
      }
    }
  }
  super_beg[nsup] = (int)chains.size();
  if ((int64_t)codes.size() > INT32_MAX) {
    record_error("streamed sweep: more than 2^31-1 entries");
    return BSP_INVALID;
  }
  S.n_super = nsup;
  S.n_chains = nc;
  S.super_beg = std::move(super_beg);
  S.chains = std::move(chains);
  S.rec = std::move(rec);
  S.codes = std::move(codes);
  S.src_blk = std::move(src);
  S.q_row = std::move(q_row);
  S.ent_q = std::move(ent_q);
  return BSP_OK;
}

int stream_build(int n, bool ascending, int warps, const SweepEntries& E, bool trans_blocks, bool has_d,
                 bool trans_d, StreamSym& S) {
  StreamPlan P;
  BSP_TRY(stream_plan(n, ascending, warps, E, P));
  S.n = P.n;
  S.n_super = P.n_super;
  S.n_chains = P.n_chains;
  S.W = P.W;
  S.dir = P.dir;
  S.n_levels = P.n_levels;
  S.stride = P.stride;
  S.n_ent = (int64_t)P.codes.size();
  S.trans_blocks = trans_blocks;
  S.has_d = has_d;
  S.trans_d = trans_d;
  BSP_TRY(upload_vec(S.super_beg, P.super_beg));
  BSP_TRY(upload_vec(S.chains, P.chains));
  BSP_TRY(upload_vec(S.rec, P.rec));
  BSP_TRY(upload_vec(S.codes, P.codes));
  BSP_TRY(upload_vec(S.src_blk, P.src_blk));
  BSP_TRY(upload_vec(S.q_row, P.q_row));
  BSP_TRY(upload_vec(S.ent_q, P.ent_q));
  return BSP_OK;
}

static size_t prec_bytes(int prec) { return prec == BSP_PREC_F64 ? 8 : prec == BSP_PREC_F32 ? 4 : 2; }

size_t stream_val_bytes(const StreamSym& S, int bs, int prec) {
  return (size_t)std::max<int64_t>(S.n_ent, 1) * bs * bs * prec_bytes(prec);
}
size_t stream_dval_bytes(const StreamSym& S, int bs, int prec) {
  return S.has_d ? (size_t)std::max(S.n, 1) * bs * bs * prec_bytes(prec) : 0;
}

template <typename VT>
static int gather_typed(bsp_handle_s* h, const StreamSym& S, int bs, const double* fvals, const double* dinv,
                        StreamVals& out) {
  const int64_t b2 = (int64_t)bs * bs;
  const size_t vb = (size_t)std::max<int64_t>(S.n_ent, 1) * b2 * sizeof(VT);
  if (out.vals.n < vb) BSP_TRY(out.vals.alloc(vb));
  if (S.n_ent > 0) {
    if (S.has_d)
      bsp::count_launch(), k_stream_gather_premul<VT><<<grid_for(h, S.n_ent * b2, 256), 256, 0, h->stream>>>(
          S.n_ent, bs, S.src_blk.get(), S.ent_q.get(), S.q_row.get(), fvals, dinv, S.trans_blocks ? 1 : 0,
          S.trans_d ? 1 : 0, reinterpret_cast<VT*>(out.vals.get()));
    else
      bsp::count_launch(), k_stream_gather<VT, int64_t><<<grid_for(h, S.n_ent * b2, 256), 256, 0, h->stream>>>(
          S.n_ent, bs, S.src_blk.get(), fvals, S.trans_blocks ? 1 : 0, reinterpret_cast<VT*>(out.vals.get()));
  }
  if (S.has_d) {
    const size_t db = (size_t)std::max(S.n, 1) * b2 * sizeof(VT);
    if (out.dvals.n < db) BSP_TRY(out.dvals.alloc(db));
    if (S.n > 0)
      bsp::count_launch(), k_stream_gather<VT, int><<<grid_for(h, (int64_t)S.n * b2, 256), 256, 0, h->stream>>>(
          S.n, bs, S.q_row.get(), dinv, S.trans_d ? 1 : 0, reinterpret_cast<VT*>(out.dvals.get()));
  }
  BSP_CUDA_TRY(cudaPeekAtLastError());
  out.valid = true;
  return BSP_OK;
}

int stream_gather(bsp_handle_s* h, const StreamSym& S, int bs, int prec, const double* fvals,
                  const double* dinv, StreamVals& out) {
  if (prec == BSP_PREC_F64) return gather_typed<double>(h, S, bs, fvals, dinv, out);
  if (prec == BSP_PREC_F32) return gather_typed<float>(h, S, bs, fvals, dinv, out);
  return gather_typed<__nv_bfloat16>(h, S, bs, fvals, dinv, out);
}

// ------------------------------------------------------------------ host: launch
template <int BS, typename VT, bool HAS_D, int W, int DEPTH>
static int launch_ss(bsp_handle_s* h, const SSP<VT>& p) {
  constexpr size_t smem = SSCfg<BS, VT, HAS_D, W, DEPTH>::kSmem;
  static int per_sm = 0;
  if (!per_sm) {
    auto kern = k_ssweep<BS, VT, HAS_D, W, DEPTH>;
    BSP_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int b = 0;
    BSP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kern, W * 32, smem));
    per_sm = std::max(1, b);
  }
  const int grid = std::min(h->num_sms * per_sm, std::max(1, p.n_super));
  bsp::count_launch(), k_ssweep<BS, VT, HAS_D, W, DEPTH><<<grid, W * 32, smem, h->stream>>>(p);
  BSP_CUDA_TRY(cudaPeekAtLastError());
  return BSP_OK;
}

// Warps per CTA and ring depth of a configuration: the deepest ring (at most
// 4 rows) that keeps two CTAs on an SM, else the deepest for one CTA.
template <int BS, typename VT, bool HAS_D> struct SSPick {
  static constexpr int W = BS >= 16 ? 4 : 16;  // the layout's grouping depends on BS only
  static constexpr size_t sm(int d) {
    return d == 4 ? SSCfg<BS, VT, HAS_D, W, 4>::kSmem : d == 3 ? SSCfg<BS, VT, HAS_D, W, 3>::kSmem
                                                                 : SSCfg<BS, VT, HAS_D, W, 2>::kSmem;
  }
  static constexpr size_t kTwo = 110 * 1024, kOne = 220 * 1024;
  static constexpr int DEPTH = sm(4) <= kTwo ? 4 : sm(3) <= kTwo ? 3 : sm(4) <= kOne ? 4 : sm(3) <= kOne ? 3 : 2;
  static_assert(sm(DEPTH) <= kOne, "streamed sweep staging does not fit shared memory");
};

template <int BS, typename VT>
static int launch_bs(bsp_handle_s* h, const StreamSym& S, const SSP<VT>& p) {
  if (S.W != SSPick<BS, VT, true>::W) {
    record_error("streamed sweep: layout built for a different warp count");
    return BSP_INVALID;
  }
  if (S.has_d) return launch_ss<BS, VT, true, SSPick<BS, VT, true>::W, SSPick<BS, VT, true>::DEPTH>(h, p);
  return launch_ss<BS, VT, false, SSPick<BS, VT, false>::W, SSPick<BS, VT, false>::DEPTH>(h, p);
}

template <typename VT>
static int sweep_typed(bsp_handle_s* h, const StreamSym& S, int bs, const StreamVals& V, const double* rhs,
                       double* x, unsigned* ticket) {
  SSP<VT> p{};
  p.n_super = S.n_super;
  p.super_beg = S.super_beg.get();
  p.chains = S.chains.get();
  p.rec = S.rec.get();
  p.codes = S.codes.get();
  p.vals = reinterpret_cast<const VT*>(V.vals.get());
  p.dvals = reinterpret_cast<const VT*>(V.dvals.get());
  p.rhs = rhs;
  p.x = x;
  p.dir = S.dir;
  p.spin_limit = h->spin_limit;
  p.ticket = ticket;
  p.st = h->ws.status.get();
  BSP_CUDA_TRY(cudaMemsetAsync(ticket, 0, sizeof(unsigned), h->stream));
  if (bs == 8) return launch_bs<8, VT>(h, S, p);
  if (bs == 16) return launch_bs<16, VT>(h, S, p);
  record_error("streamed sweep: unsupported block size");
  return BSP_INVALID;
}

int stream_sweep(bsp_handle_s* h, const StreamSym& S, int bs, int prec, const StreamVals& V, const double* rhs,
                 double* x, unsigned* ticket) {
  if (!V.valid) {
    record_error("streamed sweep: values not gathered");
    return BSP_INVALID;
  }
  if (prec == BSP_PREC_F64) return sweep_typed<double>(h, S, bs, V, rhs, x, ticket);
  if (prec == BSP_PREC_F32) return sweep_typed<float>(h, S, bs, V, rhs, x, ticket);
  return sweep_typed<__nv_bfloat16>(h, S, bs, V, rhs, x, ticket);
}

}  // namespace bsp
