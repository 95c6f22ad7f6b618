/*
 * blocksp_b200.h — C ABI of the B200-native BlockSp solve path.
 *
 * Every entry point takes plain pointers and sizes, returns an int status
 * (BSP_OK == 0) and never aborts the process.  Compute runs on the GPU only:
 * there is no CPU fallback, and every call fails with BSP_NO_DEVICE when no
 * CUDA device is present.
 *
 * Conventions shared with the reference library (BlockSp v1.0):
 *   - A block-sparse matrix is block CSR: n_rows block rows, block size bs,
 *     row_ptr[n_rows+1], col_idx[nnzb], vals[nnzb*bs*bs].  Each bs x bs block is
 *     stored row-major, as blitz::TinyMatrix<T,N,N>::data() is
 *     (blocksp_containers.hpp:52-53, blocksp_dense_multiply.hpp:65).
 *     Columns inside a row may appear in any order (the reference keeps
 *     insertion order, blocksp_containers.hpp:156-163); each column at most once.
 *   - A vector with n elements, block size B and D dimensions is n*B*D
 *     contiguous values in (element, dim, b) order, which is the memory layout
 *     of solArray<T,B,D> (blocksp_containers.hpp:581) and of util::tvConcat
 *     (blocksp_utility.hpp:257-265).
 *   - "Coupled" bsmv multiplies BlockSp<T,B*D> by solArray<T,B,D>
 *     (blocksp_multiply.hpp:209-246); "multi-RHS" bsmv multiplies BlockSp<T,B>
 *     by solArray<T,B,D> dimension by dimension (blocksp_multiply.hpp:170-205).
 *
 * Functions whose name ends in _dev take device pointers and run
 * stream-ordered on the handle's stream; the others take host buffers and
 * copy them in and out (the drop-in path used by solve(A, b)).
 */
#ifndef BLOCKSP_B200_H
#define BLOCKSP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BSP_ABI_VERSION 1

/* ---- status codes (the reference ignores LAPACK info and calls std::exit
 *      on a singular diagonal, blocksp_preconditioners.hpp:47-51; here every
 *      failure is returned) ---- */
enum bsp_status {
  BSP_OK = 0,
  BSP_ZERO_PIVOT = 1,    /* singular diagonal block in Diag/SOR/ILU0          */
  BSP_NOT_SPD = 2,       /* non-positive pivot in the IChol0 block Cholesky    */
  BSP_BREAKDOWN = 3,     /* Krylov breakdown (p'Ap <= 0 in pCG, H(j+1,j)=0 ...) */
  BSP_MAXIT = 4,         /* iteration limit reached before the tolerance      */
  BSP_NAN = 5,           /* NaN or Inf met in a residual                      */
  BSP_TIMEOUT = 6,       /* a bounded device-side wait gave up                */
  BSP_CUDA_ERROR = 7,    /* a CUDA runtime call failed                        */
  BSP_INVALID = 8,       /* bad argument (size, pointer, unsupported shape)   */
  BSP_NO_DEVICE = 9,     /* no CUDA device visible                            */
  BSP_OUT_OF_MEMORY = 10
};

/* Stored copy of the matrix a bsmv reads, and its vector type:
 * BSP_F64 FP64 blocks and vectors; BSP_F32 FP32 blocks and vectors; BSP_BF16 BF16
 * blocks with FP32 vectors; BSP_F32_STORE / BSP_BF16_STORE FP32 / BF16 blocks with
 * FP64 vectors and FP64 accumulation (the mixed-precision inner operator). */
enum bsp_dtype { BSP_F64 = 0, BSP_F32 = 1, BSP_BF16 = 2, BSP_F32_STORE = 3, BSP_BF16_STORE = 4 };

/* Preconditioner kinds (blocksp_preconditioners.hpp:66-538). */
enum bsp_precond_kind {
  BSP_PC_NONE = 0,       /* NoPre, :66-71                                     */
  BSP_PC_DIAG_LU = 1,    /* Diag<dense::LUFactor>, :75-111                    */
  BSP_PC_DIAG_CHOL = 2,  /* Diag<dense::CholeskyFactor>, :75-111              */
  BSP_PC_SOR_LU = 3,     /* SOR<dense::LUFactor> (SOR_pGMRES), :116-240       */
  BSP_PC_SOR_CHOL = 4,   /* SOR<dense::CholeskyFactor> (SOR_pCG), :116-240    */
  BSP_PC_ILU0 = 5,       /* ILU0, :246-357                                    */
  BSP_PC_ICHOL0 = 6,     /* IChol0, :364-538                                  */
  BSP_PC_LEARNED_LLT = 7,/* learned factor L, applied as L L^T (no reference) */
  BSP_PC_LEARNED_LU = 8  /* learned factors L,U, applied as (LU) (no reference) */
};

/* Arithmetic of the inner work (bsmv + preconditioner apply). */
enum bsp_precision {
  BSP_PREC_F64 = 0,      /* everything in FP64: the reference's method         */
  BSP_PREC_F32 = 1,      /* FP32 bsmv/apply inside FP64 iterative refinement   */
  BSP_PREC_BF16 = 2      /* BF16 storage, FP32 accumulate, inside FP64 IR      */
};

/* Stopping rule. */
enum bsp_stop_rule {
  BSP_STOP_REFERENCE = 0,  /* the reference's own test: pCG compares the
                              recursive ||r|| with tol*||M^-1 b||
                              (blocksp_solvers.hpp:61-69); pGMRES compares the
                              preconditioned least-squares residual with
                              tol*||M^-1 b|| (blocksp_solvers.hpp:167-232)     */
  BSP_STOP_TRUE_RESIDUAL = 1 /* FP64 true residual ||b-Ax||/||b|| <= tol       */
};

typedef struct bsp_handle_s* bsp_handle_t;
typedef struct bsp_matrix_s* bsp_matrix_t;
typedef struct bsp_precond_s* bsp_precond_t;

typedef struct {
  int kind;            /* bsp_precond_kind                                     */
  double sor_w;        /* SOR damping w (reference default 1.6, solvers.hpp:363) */
  int sor_nu;          /* sweeps per direction (default 3)                      */
  int sor_type;        /* <0 backward only, 0 symmetric, >0 forward only        */
  int precision;       /* bsp_precision of the stored factors                  */
} bsp_precond_params;

typedef struct {
  double tol;          /* relative tolerance                                   */
  int max_iters;       /* maxIters (pCG default 1000, pGMRES 500, structs 5000) */
  int restart;         /* pGMRES restart length, <0 = never (solvers.hpp:239)   */
  int k;               /* deflated-restart size k (deflated_restart.hpp:38)     */
  int print_iters;     /* print "pCG iters N" / "pGMRES iters N"                */
  int stop_rule;       /* bsp_stop_rule                                         */
  int precision;       /* bsp_precision of the inner work                       */
  double inner_tol;    /* mixed precision: relative tolerance of each inner solve */
  int max_outer;       /* mixed precision: max refinement steps                 */
  int print_eig_info;  /* pGMRES: print the Ritz (harmonic Ritz if restarted)
                          value summary of the final H (solvers.hpp:272-288)    */
} bsp_solve_opts;

typedef struct {
  int status;          /* bsp_status of the solve                              */
  int iters;           /* the reference's printed count ("pCG iters N")        */
  int n_hist;          /* entries written to the residual history              */
  int n_restarts;      /* pGMRES restarts performed                             */
  int n_outer;         /* mixed precision: refinement steps taken               */
  int inner_iters;     /* mixed precision: total inner iterations               */
  double res0;         /* ||M^-1 b||, the reference's res_mag[0]                */
  double final_res;    /* last history entry                                    */
  double true_rel_res; /* FP64 ||b - A x|| / ||b|| computed on the GPU         */
  double setup_ms;     /* preconditioner build time (device events)           */
  double solve_ms;     /* solve time (device events)                            */
} bsp_solve_info;

/* ---------------- handle ---------------- */
/* One handle per CUDA stream; a handle is not thread-safe (the reference is
 * single-threaded, blocksp_solvers.hpp has no synchronisation). stream may be
 * NULL (the handle creates its own non-blocking stream). */
int bsp_handle_create(int device, void* stream, bsp_handle_t* out);
int bsp_handle_destroy(bsp_handle_t h);
int bsp_handle_sync(bsp_handle_t h);
void* bsp_handle_stream(bsp_handle_t h);
/* Device memory the library caches (no counterpart in the reference, which
 * allocates on the host).  Buffers the library frees (matrices,
 * preconditioners, handle scratch) are kept per device, up to 32 GiB, and
 * reused by later allocations of nearly the same size, so repeated set-up
 * avoids cudaMalloc / cudaFree.  Release returns the cache of `device` (-1:
 * every device) to the driver; the allocator also does so by itself before
 * it reports an allocation failure.  The symbolic analyses of the last four
 * sparsity patterns (level schedules, sweep layouts, elimination plans) are
 * kept the same way: a matrix created with a pattern seen before — a new time
 * step, a Newton update — reuses them instead of analysing it again; release
 * drops them as well. */
int bsp_release_cached_memory(int device);
int bsp_cached_memory(int device, int64_t* bytes);
/* Failure detection (no counterpart in the reference, which never waits on
 * another thread): every device-side wait of the sync-free sweeps and
 * factorisations polls at most `polls` times (default 2^22, with a nanosleep
 * back-off) before it gives up, records BSP_TIMEOUT with the block row, and
 * returns; the launch then completes and the call reports BSP_TIMEOUT.  A
 * small value makes the waits of a large sweep run out on purpose (tests).
 * Applies to launches made after the call; polls >= 1. */
int bsp_handle_set_spin_limit(bsp_handle_t h, unsigned polls);
const char* bsp_status_string(int status);
const char* bsp_last_error(bsp_handle_t h);
int bsp_device_count(int* count);
int bsp_abi_version(void);
/* Number of CUDA kernels this library has launched in this process (all
 * handles and threads); a diagnostic for benchmarks and tests. */
uint64_t bsp_launch_count(void);

/* ---------------- matrix ----------------
 * Replaces the packing of BlockSp<T,N> = Sp::CSR<TinyMatrix<T,N,N>>
 * (blocksp_containers.hpp:52-53, 92-496): the caller hands over the CSR arrays
 * once; the handle keeps the device copy.  vals are FP64; lower-precision
 * copies are made on demand for mixed precision. */
int bsp_matrix_create(bsp_handle_t h, int n_rows, int n_cols, int bs, int64_t nnzb,
                      const int* row_ptr, const int* col_idx, const double* vals,
                      bsp_matrix_t* out);
/* Same, from arrays already in device memory (copied). */
int bsp_matrix_create_dev(bsp_handle_t h, int n_rows, int n_cols, int bs, int64_t nnzb,
                          const int* d_row_ptr, const int* d_col_idx, const double* d_vals,
                          bsp_matrix_t* out);
/* Complex T = std::complex<double> (BlockSp<std::complex<double>, N>): vals
 * holds nnzb complex bs x bs row-major blocks as interleaved (re, im) doubles.
 * The matrix is kept as its real embedding (complex entry ar + i ai ->
 * [[ar, -ai], [ai, ar]]), so bsp_matrix_info reports block size 2 bs, and a
 * complex vector (interleaved doubles, the std::complex<double> layout) is a
 * vector of 2 n bs doubles for every call on it: bsmv computes the complex
 * product; Diag / SOR / ILU0 preconditioners are the complex ones; pGMRES
 * (bsp_pgmres, bsp_pgmres_dev) runs in complex arithmetic, FP64 with the
 * reference's stopping rule.  IChol0, pCG and the learned preconditioner are
 * real only (BSP_INVALID), as in the reference (blocksp_solvers.hpp:55, 485).
 * bs <= 16. */
int bsp_matrix_create_complex(bsp_handle_t h, int n_rows, int n_cols, int bs, int64_t nnzb,
                              const int* row_ptr, const int* col_idx, const double* vals,
                              bsp_matrix_t* out);
/* complex block size of a complex matrix, 0 for a real one */
int bsp_matrix_complex_bs(bsp_matrix_t A, int* complex_bs);
int bsp_matrix_destroy(bsp_matrix_t A);
int bsp_matrix_info(bsp_matrix_t A, int* n_rows, int* n_cols, int* bs, int64_t* nnzb);
/* Device pointers of the packed matrix (row_ptr, col_idx, FP64 vals). */
int bsp_matrix_device_ptrs(bsp_matrix_t A, const int** row_ptr, const int** col_idx,
                           const double** vals);
/* Build the FP32 or BF16 copy of the values (idempotent). */
int bsp_matrix_make_lowp(bsp_matrix_t A, int dtype);

/* ---------------- bsmv ----------------
 * y = alpha * op(A) * x + beta * z   (z may alias y; z == NULL means 0)
 * nrhs == 1: BlockSp<T,N> x solArray with N = bs (coupled form when the
 *            solArray has D > 1 and N = B*D; blocksp_multiply.hpp:209-246).
 * nrhs == D > 1: BlockSp<T,B> x solArray<T,B,D>, the same block applied to
 *            each dimension (blocksp_multiply.hpp:170-205, 252-285).
 * transpose != 0: op(A) = A^T (blocksp_multiply.hpp:196-204, 280-284).
 * The reference's void bsmv(b, A, x) (multiply.hpp:386-390, accumulating)
 * is alpha = 1, beta = 1, z = y; bsmv(A, x) returning a new array is beta = 0.
 * dtype selects the stored copy of A and the vector type (enum bsp_dtype); the
 * low-precision copies must exist (bsp_matrix_make_lowp). */
int bsp_bsmv_dev(bsp_handle_t h, bsp_matrix_t A, int nrhs, int transpose, int dtype,
                 double alpha, const void* x, double beta, const void* z, void* y);
/* Host-buffer form (FP64): copies x (and y when beta != 0) in, y out. */
int bsp_bsmv(bsp_handle_t h, bsp_matrix_t A, int nrhs, int transpose,
             double alpha, const double* x, double beta, double* y);

/* ---------------- vector reductions (FP64, deterministic) ----------------
 * dot (blocksp_containers.hpp:974-996), twoNorm (998-1012), axpy (857-864). */
int bsp_dot_dev(bsp_handle_t h, int64_t n, const double* x, const double* y, double* out_dev);
int bsp_dot(bsp_handle_t h, int64_t n, const double* x_dev, const double* y_dev, double* out_host);
int bsp_axpy_dev(bsp_handle_t h, int64_t n, double a, const double* x, double* y);
/* FP64 dot product that allocates nothing; no counterpart in the reference.
 * For callers that cannot call cudaMalloc where they need the result (code
 * handed a stream and device pointers by a framework that owns the
 * allocator), so cannot create a handle.  Stream-ordered on `stream` on the
 * current device; writes the result to out_dev.  Scratch is a fixed device
 * array (about 32 KiB per GPU, held until exit): n is limited to 33,554,432
 * elements and larger n returns BSP_INVALID.  The first call on a device
 * resolves the scratch address (cudaGetSymbolAddress), so make it before any
 * stream capture.  The resolved address is kept for the life of the
 * process: after cudaDeviceReset (or anything else that destroys the
 * device's primary context) it is stale, so do not call this function on a
 * device again after resetting it.  Calls share the scratch: calls that
 * overlap on the GPU race, so serialise them (one stream, or events). */
int bsp_dot_noalloc(void* stream, int64_t n, const double* x, const double* y, double* out_dev);

/* ---------------- preconditioners ----------------
 * Construction = the reference constructor: makeADInv (preconditioners.hpp:22-63),
 * ILU0::factor (:274-291), IChol0::factor (:393-429).  A must outlive pc, as
 * A_Ptr must in the reference (:80, :120). */
int bsp_precond_create(bsp_handle_t h, bsp_matrix_t A, const bsp_precond_params* params,
                       bsp_precond_t* out);
int bsp_precond_destroy(bsp_precond_t pc);
/* r <- M^{-1} r in place, as operator()(solArray&) (preconditioners.hpp:541-556).
 * nrhs as for bsmv (1 unless the matrix is BlockSp<T,B> with D dims). */
int bsp_precond_apply_dev(bsp_handle_t h, bsp_precond_t pc, double* r);
int bsp_precond_apply(bsp_handle_t h, bsp_precond_t pc, double* r_host);
/* Copy the factored blocks back (ILU0: LU in A's layout; IChol0: L in the
 * layout of A.lowTri(); Diag/SOR: inverted diagonal blocks, n*bs*bs). */
int bsp_precond_export(bsp_precond_t pc, double* vals_host, int64_t capacity);
int bsp_precond_info(bsp_precond_t pc, int* kind, int* n_levels_lower, int* n_levels_upper,
                     int64_t* factor_nnzb);

/* ---------------- Krylov solvers ----------------
 * pCG  (blocksp_solvers.hpp:51-105)  and  pGMRES with Morgan deflated restart
 * (blocksp_solvers.hpp:156-295, blocksp_deflated_restart.hpp:38-269).
 * pc may be NULL (NoPre).  x is the output (the reference starts from x = 0).
 * hist (host, may be NULL) receives up to hist_cap residual magnitudes: the
 * reference's res_mag sequence.  b, x are device pointers for _dev. */
int bsp_pcg_dev(bsp_handle_t h, bsp_matrix_t A, bsp_precond_t pc, const double* b, double* x,
                const bsp_solve_opts* opts, double* hist, int hist_cap, bsp_solve_info* info);
int bsp_pgmres_dev(bsp_handle_t h, bsp_matrix_t A, bsp_precond_t pc, const double* b, double* x,
                   const bsp_solve_opts* opts, double* hist, int hist_cap, bsp_solve_info* info);
/* Host-buffer forms: upload b, solve, download x (solve(A,b) of the solver
 * structs, solvers.hpp:378-381, 422-425, 455-458, 489-492). */
int bsp_pcg(bsp_handle_t h, bsp_matrix_t A, bsp_precond_t pc, const double* b, double* x,
            const bsp_solve_opts* opts, double* hist, int hist_cap, bsp_solve_info* info);
int bsp_pgmres(bsp_handle_t h, bsp_matrix_t A, bsp_precond_t pc, const double* b, double* x,
               const bsp_solve_opts* opts, double* hist, int hist_cap, bsp_solve_info* info);
/* FP64 true relative residual ||b - A x|| / ||b|| on the device. */
int bsp_true_residual_dev(bsp_handle_t h, bsp_matrix_t A, const double* b, const double* x,
                          double* rel_res_host);

/* ---- batched solver -------------------------------------------------------
 * Many independent SPD systems (block sizes 4, 8 or 16, uneven sizes), each
 * with nrhs right-hand sides, solved by block-IChol0 pCG.  Replaces the loop
 *     for each system s, for each RHS d:
 *         x[s][d] = IChol0_pCG<T,bs,1>(A_s, tol, maxIters).solve(A_s, b[s][d])
 * (blocksp_solvers.hpp:481-492 with pCG :51-105 and IChol0
 * blocksp_preconditioners.hpp:364-536); no single reference call computes it,
 * because the reference pCG couples the D dims of a solArray<T,B,D> through
 * one alpha/beta.  Every (system, RHS) pair keeps its own alpha, beta,
 * stopping test and iteration count.
 *
 * Packed inputs: systems in order; row_ptr holds each system's n_rows[s]+1
 * entries (starting at 0), col_idx and vals each system's nnzb[s] blocks
 * (local column indices; bs[s] x bs[s] row-major FP64 blocks).
 * Vectors (b, x): systems in order, each n_rows[s] x nrhs x bs[s] doubles in
 * the solArray<T,bs,nrhs> (element, RHS, component) order. */
typedef struct bsp_batch_s* bsp_batch_t;

typedef struct {
  double tol;       /* relative tolerance of every pair (reference pCG rule) */
  int max_iters;    /* per pair, as pCG's maxIters */
  int mode;         /* 0: one graph launch with a device-side loop; 1: the
                       iteration graph replayed by the host */
  int check_every;  /* mode 1: iterations between status reads */
  int hist_cap;     /* residual-history entries kept per pair (0: none) */
  int retune;       /* 1: re-run the launch-shape autotuner */
} bsp_batch_opts;

typedef struct {
  int status;           /* BSP_OK when every pair converged */
  int n_pairs;          /* systems x nrhs */
  int n_converged;
  int iters_max;        /* most pCG iterations of any pair */
  long long iters_total;
  int graph_iters;      /* iterations the batched loop executed */
  double setup_ms;      /* autotune + graph capture (0 when reused) */
  double solve_ms;      /* device time of the solve */
} bsp_batch_info;

int bsp_batch_create(bsp_handle_t h, int n_sys, const int* n_rows, const int* bs, const int64_t* nnzb,
                     const int* row_ptr, const int* col_idx, const double* vals, bsp_batch_t* out);
int bsp_batch_destroy(bsp_batch_t B);
/* Per group of equal block size: its block size, systems, rows and the launch
 * shapes the autotuner chose (0 before the first solve).  Arrays hold up to 4. */
int bsp_batch_tuning(bsp_batch_t B, int* n_groups, int* group_bs, int* group_systems, int64_t* group_rows,
                     int* tile_threads, int* tile_ctas_per_sm, int* sweep_ctas_per_sm);
int bsp_batch_pcg_dev(bsp_handle_t h, bsp_batch_t B, int nrhs, const double* b, double* x,
                      const bsp_batch_opts* opts, bsp_batch_info* info);
int bsp_batch_pcg(bsp_handle_t h, bsp_batch_t B, int nrhs, const double* b_host, double* x_host,
                  const bsp_batch_opts* opts, bsp_batch_info* info);
/* Per-pair results of the last solve, indexed [system * nrhs + rhs]: pCG
 * iterations, state (1 converged, 2 max iterations, 4 NaN), last residual and
 * (hist_cap > 0) the residual history, hist_cap entries per pair. */
int bsp_batch_results(bsp_batch_t B, int nrhs, int* iters, int* state, double* final_res, double* hist,
                      int hist_cap);

/* ---- learned preconditioner ------------------------------------------------
 * No reference counterpart.  A message-passing network over the block graph
 * of A (nodes = block rows, edges = off-diagonal blocks; hidden width 32,
 * 3 layers; 8x8 blocks) emits a correction dF with A's sparsity to the
 * block-ILU0 factors; M = L U is stored in the ILU0 structures
 * (BSP_PC_LEARNED_LU) and applied by the same triangular sweeps.  The network
 * is trained on the GPU with this library's own forward/backward kernels on
 *   loss = (1/K) sum_k ||M^-1 A q_k - q_k||^2,
 * q_k the orthonormal Arnoldi vectors of the ILU0-preconditioned operator
 * from M0^-1 b (its gradient uses M^-1 and M^-T, both by triangular sweeps).
 * Parameters are packed per layer as W (out x in, row-major) then b, in the
 * order encoder-node, encoder-edge, (message, update) x 3, decoder-edge,
 * decoder-diagonal.  dtype BSP_F32 trains/infers in FP32, BSP_F64 in FP64. */
typedef struct bsp_learned_s* bsp_learned_t;

int bsp_learned_create(bsp_handle_t h, int bs, int dtype, bsp_learned_t* out);
/* Factor form the network emits (default BSP_LEARNED_LU): BSP_LEARNED_LU
 * corrects the block-ILU0 factors (M = L U, pGMRES, BSP_PC_LEARNED_LU);
 * BSP_LEARNED_LLT corrects the block-IChol0 factor (M = L L^T, SPD, pCG,
 * BSP_PC_LEARNED_LLT; lower blocks only, diagonal corrections kept lower
 * triangular).  loss_grad then takes an IChol0 preconditioner in place of
 * ILU0.  No counterpart in the reference. */
enum bsp_learned_form { BSP_LEARNED_LU = 0, BSP_LEARNED_LLT = 1 };
int bsp_learned_set_form(bsp_learned_t M, int form);
/* Relaxation of the learned factors (default 0): the off-diagonal blocks of the
 * block-ILU0 / block-IChol0 factors are scaled by 1 + relax before the
 * network's correction is added (a modified-incomplete-factorisation-like
 * compensation), in bsp_learned_loss_grad and bsp_learned_precond alike.
 * relax must lie in (-1, 4).  No counterpart in the reference. */
int bsp_learned_set_relax(bsp_learned_t M, double relax);
int bsp_learned_get_relax(bsp_learned_t M, double* relax);
int bsp_learned_destroy(bsp_learned_t M);
int bsp_learned_param_count(bsp_learned_t M, int64_t* count);
int bsp_learned_set_params(bsp_learned_t M, const double* params, int64_t count);
int bsp_learned_get_params(bsp_learned_t M, double* params, int64_t count);
/* gradient of the last bsp_learned_loss_grad call */
int bsp_learned_get_grads(bsp_learned_t M, double* grads, int64_t count);
/* dF (device, nnzb*bs*bs, A's block order) for the current parameters */
int bsp_learned_forward(bsp_handle_t h, bsp_learned_t M, bsp_matrix_t A, double* dF);
/* ILU0 factors of an ILU0 preconditioner in A's block order (device) */
int bsp_learned_ilu_factors(bsp_handle_t h, bsp_precond_t ilu, double* F0);
/* loss for the factors of `ilu` (BSP_PC_ILU0 on A) plus dF, over probes
 * (device, K orthonormal vectors of n*bs); keeps the parameter gradient */
int bsp_learned_loss_grad(bsp_handle_t h, bsp_learned_t M, bsp_matrix_t A, bsp_precond_t ilu, int n_probes,
                          const double* probes, double* loss);
int bsp_learned_adam_step(bsp_handle_t h, bsp_learned_t M, double lr, double beta1, double beta2, double eps);
/* K orthonormal Arnoldi vectors of M^-1 A from M^-1 b (device; pc may be NULL) */
int bsp_learned_probes(bsp_handle_t h, bsp_matrix_t A, bsp_precond_t pc, const double* b, int K,
                       double* probes);
/* In place on K device vectors (n*bs each): `steps` iterations of
 * e <- e - M^-1 A e (the error of the preconditioned stationary iteration,
 * which keeps the slow modes), then orthonormalisation. */
int bsp_learned_smooth(bsp_handle_t h, bsp_matrix_t A, bsp_precond_t pc, int K, int steps, double* vecs);
/* Builds the learned preconditioner of A (ILU0 + network correction). */
int bsp_learned_precond(bsp_handle_t h, bsp_learned_t M, bsp_matrix_t A, int precision, bsp_precond_t* out);

/* ---------------- eigenvalue diagnostics ----------------
 * arnoldi_eigenvalues (blocksp_solvers.hpp:306-334) with Eigenvalues_Arr
 * (blocksp_dense_solvers.hpp:909-1000): `iters` Arnoldi steps of M^-1 A (pc
 * may be NULL) from q_0 = e_0 on the GPU, then the eigenvalues of the square
 * part of H (harmonic Ritz values H_n + h_mn^2 H_n^-T e_n e_n^T when
 * harmonic_ritz).  wr, wi: host arrays of iters values; *n_out = the number
 * of values (fewer than iters when the Krylov space is exhausted: where the
 * reference would read past its basis, this stops).  print_info / print_vals
 * print the reference's printEigInfo / printEigVals text. */
int bsp_arnoldi_eigenvalues(bsp_handle_t h, bsp_matrix_t A, bsp_precond_t pc, int iters, int harmonic_ritz,
                            int print_info, int print_vals, double* wr, double* wi, int* n_out);

/* ---------------- block sparse matrix algebra ----------------
 * Results are new device matrices (destroy with bsp_matrix_destroy); their
 * blocks are ordered within each row as the reference's containers create
 * them (BlockSp::operator() appends a missing block at the row's end).
 * bs_id (blocksp_multiply.hpp:335-336, blkSpIdent :21-28): n x n identity. */
int bsp_bs_id(bsp_handle_t h, int n, int bs, bsp_matrix_t* out);
/* bs_tr (:339-340, blkSpTranspose :31-42): block (j, i) = A_ij^T. */
int bsp_bs_tr(bsp_handle_t h, bsp_matrix_t A, bsp_matrix_t* out);
/* bsmm (:343-362, blkSpMatMat :51-133): C = A B, or A^T B when a_transpose;
 * each C block sums its block products in the reference's order.  Triple and
 * quadruple products nest to the right (:137-159). */
int bsp_bsmm(bsp_handle_t h, bsp_matrix_t A, bsp_matrix_t B, int a_transpose, bsp_matrix_t* out);
/* C = alpha A + beta B (CSR::operator+= / -= / *=, blocksp_containers.hpp:
 * 302-318, 340-347): A's blocks, then B's blocks missing from A per row. */
int bsp_matrix_add(bsp_handle_t h, double alpha, bsp_matrix_t A, double beta, bsp_matrix_t B,
                   bsp_matrix_t* out);
/* Structure and FP64 values back to host buffers (row_ptr[n_rows+1],
 * col_idx[nnzb], vals[nnzb*bs*bs]). */
int bsp_matrix_export(bsp_matrix_t A, int* row_ptr, int* col_idx, double* vals);

/* ---------------- MatrixMarket files ----------------
 * mtxMatrix_to_BlockSp / mtxArray_to_solArray (blocksp_tests.hpp:582-699).
 * Reading starts at 1-based line max(start_line, 1), the size line.
 * Matrix: entries "i j value" (1-based unless base_zero, which the reference
 * ignores); symmetric fills (j, i) too; blocks bs x bs in order of first
 * appearance, a repeated entry overwrites.  Call once with row_ptr == NULL
 * for n_rows, n_cols, nnzb, then with row_ptr[n_rows+1], col_idx[nnzb],
 * vals[nnzb*bs*bs].  Vector: M x 1 values in solArray<T,B,D> order (value i
 * at flat position i); B*D must divide M.  The reference misplaces values
 * for D > 1 (in-block index i % B instead of i % (B*D), :679); this reader
 * does not.  Call with out == NULL for the count. */
int bsp_mtx_read_matrix(const char* path, int bs, int start_line, int symmetric, int base_zero, int* n_rows,
                        int* n_cols, int64_t* nnzb, int* row_ptr, int* col_idx, double* vals);
int bsp_mtx_read_vector(const char* path, int start_line, int B, int D, int64_t* n_values, double* out);

#ifdef __cplusplus
}
#endif
#endif /* BLOCKSP_B200_H */
