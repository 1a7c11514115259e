/*
 * csipm.h — C ABI of the B200-native matrix-free interior-point hot path of
 * CompressedSensingIPM.jl (sparse DFT recovery from a real signal with missing
 * samples: min_beta 1/2 ||A beta - z0||^2 + lambda ||beta||_1,
 * A = P_Omega * sqrt(N) * Re(IDFT(B beta))).
 *
 * Every entry point is the replacement for one function of the reference's
 * NLPModels / MadNLP plugin surface; the reference location is given beside
 * each declaration (paths inside the CompressedSensingIPM.jl repository).
 *
 * Conventions
 *   - Arrays are column-major (dim 1 fastest) and 0-based, exactly Julia's
 *     memory layout, so a CuArray's pointer can be passed unchanged.
 *   - Vector arguments are DEVICE pointers owned by the caller (CuArray /
 *     torch / cudaMalloc memory) unless the name says host_.  The library never
 *     frees them.  Real arrays must be 16-byte aligned (CuArray/cudaMalloc
 *     memory is; a view at an even element offset is).
 *   - Complex arrays are interleaved (re, im) FP64, i.e. ComplexF64 memory.
 *   - Every function returns a csipm_status (0 = success).  No exception
 *     crosses the ABI; csipm_last_error() describes the last failure.
 *   - One handle = one CUDA stream.  Calls are stream-ordered and asynchronous
 *     except those returning a host scalar (csipm_obj, csipm_solve, ...),
 *     which synchronise the handle's stream.  A handle is not thread-safe;
 *     distinct handles may be used concurrently from different threads.
 */
#ifndef CSIPM_H
#define CSIPM_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define CSIPM_API __attribute__((visibility("default")))
#else
#define CSIPM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define CSIPM_ABI_VERSION 2

typedef enum {
    CSIPM_OK = 0,
    CSIPM_ERR_INVALID = -1,        /* bad argument (null pointer, size, misalignment) */
    CSIPM_ERR_ODD_DIM = -2,        /* a dimension is odd or < 2 (src/fft_utils.jl:130 requires even sizes) */
    CSIPM_ERR_UNSUPPORTED = -3,    /* size beyond the on-chip FFT passes */
    CSIPM_ERR_OOM = -4,            /* device allocation failed */
    CSIPM_ERR_CUDA = -5,           /* a CUDA call failed */
    CSIPM_ERR_CG_MAXITER = -6,     /* CG hit its iteration cap before the tolerance */
    CSIPM_ERR_NONFINITE = -7,      /* NaN/Inf detected in the iteration */
    CSIPM_ERR_IPM_MAXITER = -8,    /* IPM hit max_iter before the tolerance */
    CSIPM_ERR_NO_DEVICE = -9       /* no CUDA device / the library was not built for it */
} csipm_status;

typedef enum { CSIPM_FP64 = 0, CSIPM_MIXED = 1 } csipm_precision;

typedef struct csipm_handle_s* csipm_handle;

/* Problem description.  Replaces FFTParameters (src/fft_utils.jl:1-14). */
typedef struct {
    int dim;                        /* 1, 2 or 3                                 (DFTdim)  */
    int size[3];                    /* N1, N2, N3 (unused entries ignored), even (DFTsize) */
    double lambda;                  /* l1 weight                                 (lambda)  */
    const double* z0;               /* DEVICE, N reals, zero at missing samples  (z0)      */
    const int64_t* host_missing;    /* HOST, 0-based column-major linear indices of the
                                       missing samples (index_missing, 1-based in Julia),
                                       may be NULL when n_missing == 0 */
    int64_t n_missing;
} csipm_problem;

/* Options.  Mirrors the FFTNLPModel kwargs (src/fft_model.jl:12-15) and the
 * MadNLP options used by the reference drivers (test/ipm_example_1D.jl:60-70). */
typedef struct {
    int rdft;                  /* 1: real FFT / half spectrum (reference rdft=true); 0: full spectrum */
    int precision;             /* csipm_precision */
    int preconditioner;        /* 1: block-diagonal preconditioner (reference default true) */
    double tol;                /* IPM stop: relative LASSO duality gap (reference tol=1e-8) */
    int max_iter;              /* IPM iteration cap (reference max_iter=2000) */
    double cg_atol;            /* KKT solve: CG absolute tolerance (reference atol=1e-12) */
    double cg_rtol;            /* KKT solve: CG relative tolerance (reference rtol=0) */
    int cg_maxit;              /* CG iteration cap per solve */
    double ipm_cg_rtol;        /* csipm_solve: relative CG tolerance of each Newton solve */
    int ir_max;                /* mixed precision: max FP64 refinement steps per Newton solve */
    int verbose;               /* 1: print one line per IPM iteration to stderr */
    void* stream;              /* cudaStream_t every call of the handle runs on; NULL: the default stream */
    int layout;                /* csipm_solve's internal vector order: 0 (default) the half-spectrum
                                  "solver order" where the operator supports it (2D/3D), 1 the
                                  reference packing throughout.  Inputs and outputs of every entry
                                  point are in the reference packing either way. */
    int cuda_graphs;           /* 1 (default): csipm_solve runs its iterations after the first as one
                                  CUDA graph launch (a conditional while node over whole iterations,
                                  the stop test on the device, nested while nodes for the CG loops)
                                  when no Newton solve needs a host decision (FP64, or mixed with
                                  ipm_cg_rtol >= 1e-4), else each CG loop of csipm_solve /
                                  csipm_admm as one graph launch; graphs are captured once per
                                  handle; 0: plain launches (same kernels, same results) */
    int autotune;              /* 1 (default): csipm_create times the candidate launch configurations
                                  of the FFT passes for this size (two-level vs Stockham kernels,
                                  lines / rows per CTA) once per process and keeps the fastest;
                                  with the environment variable CSIPM_TUNE_CACHE naming a file, the
                                  choices persist there (one JSON object per line) and later
                                  processes start from them; 0: the built-in heuristic */
    double ipm_cg_forcing;     /* csipm_solve: forcing term of the inexact Newton solves.  Iteration k
                                  solves to min(ipm_cg_rtol, max(1e-6, ipm_cg_forcing * gap[k-1]))
                                  with gap[k-1] the previous iteration's relative duality gap, so
                                  loose solves tighten as the method converges (fixed loose solves
                                  stall once the gap is far below their accuracy); default 100,
                                  0: every solve at ipm_cg_rtol */
} csipm_options;

/* Per-solve statistics (MadNLPExecutionStats analogue + the reference's timers,
 * src/fft_utils.jl:24-25, src/fft_kkt.jl:109-110). */
typedef struct {
    int status;                /* csipm_status of the solve */
    int ipm_iter;              /* IPM iterations */
    int cg_iter;               /* total CG iterations over all Newton solves */
    int matvecs;               /* A^T A products (FP64 + FP32) */
    int refinements;           /* FP64 iterative-refinement steps (mixed precision) */
    double gap;                /* final relative LASSO duality gap */
    double obj;                /* reference objective 1/2||A b||^2 - b'A^T z0 + lambda*sum(c) (src/fft_model.jl:66-75) */
    double lasso_obj;          /* 1/2||A b - z0||^2 + lambda ||b||_1 */
    double mu;                 /* final barrier parameter (average complementarity) */
    double dual_inf;           /* final max |A^T A b - A^T z0 - z1 + z2| */
    double solve_ms;           /* wall time of csipm_solve on the device stream */
    long long launches;        /* kernels the solve launched (including early-exit CG tails) */
    int fallbacks;             /* mixed precision: Newton solves finished in FP64 after an FP32 CG breakdown */
    /* the residual pass (the solve's largest kernel: pending step, residual,
     * barrier diagonals, predictor right-hand side), timed with CUDA events on
     * the solve's stream around each launch */
    double resid_pass_ms;      /* device time of the launches the host ran (the first of a solve run
                                  with cuda_graphs; every one without) */
    double resid_pass_bytes;   /* their algorithmic bytes (vectors read + written) */
    int resid_pass_launches;   /* the launches timed */
    int graph_iters;           /* iterations run inside replays of the whole-iteration CUDA graph
                                  (cuda_graphs = 1, FP64 or mixed with ipm_cg_rtol >= 1e-4): the
                                  stop test runs on the device and the host waits once per solve */
} csipm_stats;

/* ---------------------------------------------------------------- lifecycle */

/* Fills `opt` with the reference defaults (rdft=1, FP64, preconditioner=1,
 * tol=1e-8, max_iter=2000, cg_atol=1e-12, cg_rtol=0, cg_maxit=2N). */
CSIPM_API int csipm_default_options(csipm_options* opt);

/* Builds the operator, FFT plans, mask and workspaces and computes A^T z0.
 * Replaces FFTOperator{VT}(...) (src/fft_utils.jl:16-54) together with the
 * FFTNLPModel constructor (src/fft_model.jl:12-64) and create_kkt_system
 * (src/fft_kkt.jl:113-156). */
CSIPM_API int csipm_create(const csipm_problem* prob, const csipm_options* opt, csipm_handle* out);

/* Frees everything the handle owns (never the caller's vectors). */
CSIPM_API int csipm_destroy(csipm_handle h);

/* Handles take their device memory from one stream-ordered pool per device
 * that keeps freed blocks for the next handle, so csipm_create/csipm_destroy
 * neither map memory nor synchronise the device (other handles' streams keep
 * running).  This returns the pool's unused memory to the driver (device < 0:
 * the current device).  No counterpart in the reference (CUDA.jl manages its
 * own pool). */
CSIPM_API int csipm_trim_pool(int device);

/* Message of the last failure on `h` (or of the last failed csipm_create when h is NULL). */
CSIPM_API const char* csipm_last_error(csipm_handle h);

/* N = prod(size) and the device bytes the handle holds. */
CSIPM_API int csipm_get_info(csipm_handle h, int64_t* n, size_t* device_bytes);

/* Copies the cached A^T z0 (FFTNLPModel.M_perpt_z0, src/fft_model.jl:61-62) into out (N). */
CSIPM_API int csipm_get_Atz0(csipm_handle h, double* out);

/* ---------------------------------------------------------------- mapping */

/* beta_to_DFT!(v, dim, size, beta; rdft) — src/fft_utils.jl:195-204
 * (src/mapping_cuda.jl:114-365).  Bit-exact with src/mapping_cpu_kernels.jl.
 * v: (N1/2+1)*N2*N3 complex when rdft=1, N1*N2*N3 complex when rdft=0. */
CSIPM_API int csipm_beta_to_dft(int dim, const int* size, int rdft, const double* beta, double* v, void* stream);

/* DFT_to_beta!(beta, dim, size, v) — src/fft_utils.jl:144-153
 * (src/mapping_cuda.jl:1-111).  Reads only v[1:N1/2+1, :, :]; ld1 is the
 * first-dimension extent of v (N1/2+1 for a half spectrum, N1 for a full one). */
CSIPM_API int csipm_dft_to_beta(int dim, const int* size, int ld1, const double* v, double* beta, void* stream);

/* ---------------------------------------------------------------- operator */

/* M_perp_beta: x = P_Omega(sqrt(N) Re(ifft(B beta)))  — src/fft_utils.jl:95-117.  beta, x: N. */
CSIPM_API int csipm_apply_A(csipm_handle h, const double* beta, double* x);

/* M_perpt_z: beta = B^T(fft(z)/sqrt(N)), no mask  — src/fft_utils.jl:73-93.  z, beta: N. */
CSIPM_API int csipm_apply_At(csipm_handle h, const double* z, double* beta);

/* M_perpt_M_perp_vec: y = A^T A x  — src/fft_utils.jl:67-71, 119-123.  x, y: N. */
CSIPM_API int csipm_apply_AtA(csipm_handle h, const double* x, double* y);

/* ---------------------------------------------------------------- NLPModels */

/* obj(nlp, x): 1/2||A beta||^2 - beta'A^T z0 + lambda*sum(c), x = [beta; c] (2N)
 * — src/fft_model.jl:66-75.  Synchronises; *f is a host double. */
CSIPM_API int csipm_obj(csipm_handle h, const double* x, double* f);

/* grad!(nlp, x, g): g = [A^T A beta - A^T z0; lambda] — src/fft_model.jl:77-89.  x, g: 2N. */
CSIPM_API int csipm_grad(csipm_handle h, const double* x, double* g);

/* cons!(nlp, x, c): c = [-beta - c; beta - c] — src/fft_model.jl:91-101.  x, c: 2N. */
CSIPM_API int csipm_cons(csipm_handle h, const double* x, double* c);

/* Hessian-vector product of the Lagrangian (constraints are linear):
 * hv = obj_weight * [A^T A v_beta; 0].  The reference sets hprod_available=false
 * (src/fft_model.jl:55); the same product is the A^T A block of
 * src/fft_kkt.jl:39-41.  v, hv: 2N. */
CSIPM_API int csipm_hprod(csipm_handle h, const double* v, double* hv, double obj_weight);

/* ---------------------------------------------------------------- KKT plugin */

/* build_kkt!: Lambda1 = S1 + S2, Lambda2 = S1 - S2 and the preconditioner
 * P11/P12/P22 from the slack block of pr_diag (S1 = pr_diag[2N:3N),
 * S2 = pr_diag[3N:4N)) — src/fft_kkt.jl:285-307.  pr_diag: >= 4N. */
CSIPM_API int csipm_kkt_build(csipm_handle h, const double* pr_diag);

/* mul!(y, K, x, alpha, beta) with the condensed operator
 * K = [A^T A + L1, L2; L2, L1] — src/fft_kkt.jl:27-44.  x, y: 2N. */
CSIPM_API int csipm_condensed_mul(csipm_handle h, double* y, const double* x, double alpha, double beta);

/* mul!(y, P, x, alpha, beta) with the block-diagonal preconditioner
 * — src/fft_kkt.jl:73-85.  x, y: 2N. */
CSIPM_API int csipm_precond_mul(csipm_handle h, double* y, const double* x, double alpha, double beta);

/* Body of mul!(y::KKTVector, kkt, x, alpha, beta) — src/fft_kkt.jl:223-246:
 * the 6N primal/slack/dual block [beta; c; s1; s2; y1; y2].  The caller adds
 * MadNLP's _kktmul! diagonal terms (src/fft_kkt.jl:248) itself.  x, y: 6N. */
CSIPM_API int csipm_kkt_mul(csipm_handle h, double* y, const double* x, double alpha, double beta);

/* jtprod!(y, kkt, x): y[0:4N) = J' x for the 2N constraint multipliers
 * — src/fft_kkt.jl:253-275.  x: 2N, y: >= 4N. */
CSIPM_API int csipm_jtprod(csipm_handle h, double* y, const double* x);

/* Body of solve_kkt!(kkt, w) — src/fft_kkt.jl:316-350: right-hand side
 * reduction, preconditioned CG on the condensed system (atol=cg_atol,
 * rtol=cg_rtol), back-substitution, all in place on w = [w1..w6] (6N).  The
 * caller runs MadNLP.reduce_rhs! before and finish_aug_solve! after
 * (src/fft_kkt.jl:314, 352).  Requires a prior csipm_kkt_build with the same
 * pr_diag.  *cg_iters receives the iteration count (Krylov iteration_count). */
CSIPM_API int csipm_kkt_solve(csipm_handle h, double* w, const double* pr_diag, int* cg_iters);

/* ---------------------------------------------------------------- solver */

/* The whole interior-point solve on the device (ipm_solve!,
 * src/CompressedSensingIPM.jl:31-36, with the MadNLP loop replaced by a
 * primal-dual path-following method on the same formulation and the same
 * condensed KKT operator).  beta_out (N) and, if non-NULL, c_out (N) receive
 * the solution; stats may be NULL. */
CSIPM_API int csipm_solve(csipm_handle h, double* beta_out, double* c_out, csipm_stats* stats);

/* Batched solves: advances `count` handles' interior-point solves together,
 * every step one kernel launch for all of them — the FFT passes are
 * persistent Stockham kernels over an instance table (per instance its
 * sizes, run-time plans, vector offsets, reduction workspace and control
 * block) and every element kernel runs all instances at once (gridDim.y =
 * instance).  Any sizes mix; the handles must share the dimension count,
 * whether they have missing samples, and for 1D whether the rows take the
 * long-row passes (N1/2 > 2048).  Each instance solves with its own options
 * (tol, max_iter, ipm_cg_rtol, ipm_cg_forcing, preconditioner) by
 * csipm_solve's FP64 method in the reference packing: its iterates equal
 * csipm_solve's up to the order of floating-point sums.  Runs on hs[0]'s
 * stream (the other handles' streams are joined first).  beta_out[k] (device,
 * N_k values) and stats[k] (may be NULL) receive instance k's result; returns
 * CSIPM_OK when every instance converged, else the first failure (each
 * instance's status is in its stats).  No counterpart in the reference, which
 * solves one recovery per call (src/CompressedSensingIPM.jl:31-36). */
CSIPM_API int csipm_solve_batch(csipm_handle* hs, int count, double* const* beta_out, csipm_stats* stats);

/* ---------------------------------------------------------------- timers */

/* Device time (ms, CUDA events) accumulated by the handle in the three buckets
 * the reference keeps (fft_timer / mapping_timer, src/fft_utils.jl:24-25;
 * krylov_timer, src/fft_kkt.jl:110): here operator products, elementwise
 * IPM/mapping work and CG solves.  Reset with reset != 0. */
CSIPM_API int csipm_get_timers(csipm_handle h, double* operator_ms, double* elementwise_ms, double* krylov_ms, int reset);

/* ---------------------------------------------------------------- no allocation */

/* y = A^T A x for callers that cannot allocate device memory.  No counterpart
 * in the reference: it exists for callers whose device memory is owned by a
 * pool they must not bypass (a Julia CUDA.jl or PyTorch process with a hard
 * memory limit, a serving process that pre-commits all HBM to resident
 * problems) and for loops that cannot afford cudaMalloc's implicit device
 * synchronisation.  It calls no cudaMalloc, cudaFree or allocating library
 * routine and copies nothing from the host: its scratch (the half spectrum
 * and the twiddle tables, which a small kernel writes on every call) lives in
 * one file-scope device array of 32 MiB that every GPU loading the library
 * holds until the process exits.  Problems whose half spectrum
 * ((N1/2+1)*N2*N3 complex values) and twiddle tables need more than 32 MiB —
 * above about 2.09 million complex values, e.g. 3D grids beyond 160^3; 1D
 * lengths up to 2^20 fit — are rejected with CSIPM_ERR_UNSUPPORTED and a
 * message.  The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) with that device current; make that first call
 * before any stream capture.  All calls share the array and each rewrites
 * what it reads, so calls that overlap on the GPU race: serialise them (one
 * stream, or events).  Inputs and outputs are the
 * caller's: x, y (N, device), keep_bits (device, or NULL for no missing
 * samples): one bit per sample, 1 = observed, column-major, LSB first, each
 * dim-1 row of N1 bits padded to a whole number of 32-bit words.  Runs on
 * `stream` (NULL: default stream); errors are reported by csipm_last_error(NULL). */
CSIPM_API int csipm_apply_AtA_static(int dim, const int* size, const uint32_t* keep_bits, const double* x, double* y,
                                     void* stream);

/* ---------------------------------------------------------------- Gondzio formulation */
/* GondzioNLPModel / GondzioKKTSystem (src/gondzio_model.jl, src/gondzio_kkt.jl)
 * on the same handle: beta = p - q, p, q >= 0, residual variable r,
 * x = [p; q; r] (3N), constraint z0 - A(p - q) - r = 0 (N).  The handle keeps
 * the problem's z0 pointer (FFTParameters.z0 outlives the model). */

/* NLPModels.obj: 1/2 r'r + lambda sum(p, q) — src/gondzio_model.jl:67-78 */
CSIPM_API int csipm_gondzio_obj(csipm_handle h, const double* x, double* f);
/* NLPModels.grad!: g = [lambda (2N); r] — src/gondzio_model.jl:80-93 */
CSIPM_API int csipm_gondzio_grad(csipm_handle h, const double* x, double* g);
/* NLPModels.cons!: c = z0 - A(p - q) - r — src/gondzio_model.jl:95-110 */
CSIPM_API int csipm_gondzio_cons(csipm_handle h, const double* x, double* c);
/* build_kkt!: Dp, Dq from pr_diag[0:2N) and the block preconditioner — src/gondzio_kkt.jl:278-301 */
CSIPM_API int csipm_gondzio_kkt_build(csipm_handle h, const double* pr_diag);
/* CondensedGondzioKKTSystem mul!: y = alpha [A'A + Dp, -A'A; -A'A, A'A + Dq] x + beta y (2N) — src/gondzio_kkt.jl:28-53 */
CSIPM_API int csipm_gondzio_condensed_mul(csipm_handle h, double* y, const double* x, double alpha, double beta);
/* GondzioPreconditioner mul! (2N) — src/gondzio_kkt.jl:82-93 */
CSIPM_API int csipm_gondzio_precond_mul(csipm_handle h, double* y, const double* x, double alpha, double beta);
/* MadNLP.mul! body before _kktmul!, x, y = [p; q; r; y] (4N) — src/gondzio_kkt.jl:213-248 */
CSIPM_API int csipm_gondzio_kkt_mul(csipm_handle h, double* y, const double* x, double alpha, double beta);
/* jtprod!: y = [-A'x; A'x; -x] (3N), x: N — src/gondzio_kkt.jl:250-268 */
CSIPM_API int csipm_gondzio_jtprod(csipm_handle h, double* y, const double* x);
/* solve_kkt! after MadNLP.reduce_rhs!, w = [p; q; r; y] (4N) in place; PCG
 * with the block preconditioner (cg_atol, cg_rtol) — src/gondzio_kkt.jl:303-362 */
CSIPM_API int csipm_gondzio_kkt_solve(csipm_handle h, double* w, int* cg_iters);

/* ---------------------------------------------------------------- ADMM */
typedef struct {
    int status;                /* CSIPM_OK, or CSIPM_ERR_IPM_MAXITER when maxt ran out before tol */
    int iterations;            /* ADMM iterations t */
    int cg_iter;               /* CG iterations of all x-updates */
    double err;                /* final max(|x1-x0|, |y1-y0|, |z1-z0|) */
    double solve_ms;
} csipm_admm_stats;

/* CompressedSensingADMM(fft_parameter, fft_operator; rho, maxt, tol) —
 * src/admm.jl:8-61 on the device: x0 = z = 1, y = 0; each iteration solves
 * (A'A + rho I) x = A'z0 + rho z - y by CG from zero (no preconditioner,
 * atol = rtol = sqrt(eps), cap cg_maxit), z = soft(x + y/rho, lambda/rho),
 * y += rho (x - z), until max of the three 2-norm differences <= tol.
 * z_out: N (device), the final z.  Uses the handle's IPM workspace (a later
 * csipm_solve starts afresh). */
CSIPM_API int csipm_admm(csipm_handle h, double rho, int maxt, double tol, double* z_out, csipm_admm_stats* stats);

/* ---------------------------------------------------------------- serving */
/* A request loop for many recoveries of uneven sizes (no counterpart in the
 * reference, which solves one recovery per call, src/CompressedSensingIPM.jl:31-36).
 * `slots` worker threads, each with its own CUDA stream, take requests in
 * arrival order as soon as a slot is free and the request's device footprint
 * (csipm_footprint) fits in what the admitted requests leave of `hbm_budget`;
 * a request that does not fit yet lets smaller ones behind it go first.
 * Admitted requests keep their interior-point state resident on the device
 * and their kernels overlap. */
typedef struct csipm_server_s* csipm_server;

typedef struct {
    int slots;                 /* concurrent solves; 0: 8 */
    size_t hbm_budget;         /* device bytes admitted requests may hold; 0: 80% of the free memory at create */
    int device;                /* CUDA device; -1: the current one */
    int cuda_graphs;           /* 1: each request's solve runs its iterations as one graph launch
                                  (captured per request); 0 (default): plain launches */
    int batch;                 /* > 1: a slot solves up to `batch` admitted requests of one batch
                                  class (dimension count, long-row 1D passes, missing samples or
                                  not), the closest in size to the oldest, together through
                                  csipm_solve_batch (FP64); 0 or 1 (default): one at a time */
    long long batch_max_n;     /* with batch > 1: requests of more samples are solved alone (they
                                  fill the GPU by themselves and keep their precision); 0: no limit */
} csipm_server_options;

typedef struct {
    csipm_problem problem;     /* as for csipm_create, but z0 is a HOST pointer (N reals) */
    csipm_options options;     /* from csipm_default_options, then edited; `stream` and
                                  `cuda_graphs` are ignored (each request's handle lives for one
                                  solve on its slot's stream; csipm_server_options.cuda_graphs
                                  decides for all requests) */
    double* beta_out;          /* HOST, N reals, written before the result is posted (may be NULL) */
    uint64_t tag;              /* the caller's id, returned with the result */
} csipm_request;

typedef struct {
    uint64_t tag;
    int status;                /* csipm_status of the solve */
    csipm_stats stats;
    double queue_ms;           /* submission -> admission */
    double latency_ms;         /* submission -> result posted (beta_out written) */
    size_t footprint;          /* device bytes the request was admitted with */
    char message[160];         /* the failure's message when status != 0 (truncated), else "" */
    int group;                 /* requests admitted together with this one, itself included
                                  (1: solved alone; > 1: one csipm_solve_batch) */
} csipm_result;

/* Device bytes a handle for this problem holds plus the server's staging of
 * z0 and beta (an upper bound of csipm_get_info's figure + 16N). */
CSIPM_API int csipm_footprint(int dim, const int* size, int precision, int64_t n_missing, size_t* bytes);
CSIPM_API int csipm_server_create(const csipm_server_options* opt, csipm_server* out);
/* Queues a copy of the request struct; the host buffers it points to must stay
 * valid until its result has been polled.  A slot stages z0 and beta through
 * pinned host buffers of its own, so its copies run asynchronously. */
CSIPM_API int csipm_server_submit(csipm_server s, const csipm_request* r);
/* Moves up to `max` finished results to `out` (*n of them), waiting up to
 * timeout_ms (-1: until one is ready or nothing is pending) when none is ready. */
CSIPM_API int csipm_server_poll(csipm_server s, csipm_result* out, int max, int* n, int timeout_ms);
/* Runs every queued request to completion, then frees the server. */
CSIPM_API int csipm_server_destroy(csipm_server s);

/* ---------------------------------------------------------------- diagnostics */

/* Times each kernel of one A^T A product in isolation: every pass is launched
 * `reps` times back to back between CUDA events on the handle's stream (the
 * last pass with the CG epilogue q = A^T A p + D p, p.q).  Writes up to 8
 * entries: ms_out[k] = average device ms per launch, bytes_out[k] = algorithmic
 * HBM bytes per launch (each array read or written once), name_out (optional,
 * 8 x 32 chars) = kernel role.  *npass receives the pass count (1, 3 or 5 for
 * 1D/2D/3D).  x: N, 16-byte aligned.  A CSIPM_MIXED handle times the FP32
 * passes of its CG product (x rounded to FP32).  The reference keeps only host-side timers
 * (src/fft_utils.jl:24-25); this has no counterpart there. */
CSIPM_API int csipm_profile_passes(csipm_handle h, const double* x, int reps, double* ms_out, double* bytes_out,
                                   char* name_out, int* npass);

#ifdef __cplusplus
}
#endif

#endif /* CSIPM_H */
