// Internal declarations shared by the library's translation units: the
// handle, error plumbing, launch helpers and the operator dispatch (which
// passes a product runs through for each dimension).
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/csipm.h"
#include "geometry.h"
#include "fft2.cuh"
#include "operator.cuh"
#include "solver_kernels.cuh"
#include "long1d.cuh"
#include <type_traits>

namespace csipm {
void set_last_error(const std::string& msg);
const char* get_last_error();

// Stream-ordered device memory for handles: one pool per device, created on
// first use, that keeps freed blocks for the next handle (creating and
// destroying handles then neither maps memory nor synchronises the device,
// so handles on other streams keep running).  csipm_trim_pool releases it.
cudaMemPool_t device_pool(int dev);

// Small pinned host blocks (scalar read-back slots) from a process-wide free
// list: cudaFreeHost would synchronise the device.
void* pinned_get(size_t bytes);
void pinned_put(void* p, size_t bytes);
}  // namespace csipm

namespace csipm_internal {
using namespace csipm;

inline int ew_blocks(long long n) {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    long long b = (n + EW_THREADS - 1) / EW_THREADS;
    long long cap = (long long)sms * 8;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (int)b;
}

// Grid of a grid-stride element kernel: exactly one resident wave (the SM
// count times the EW_THREADS-thread CTAs that fit on an SM with the
// kernel's registers), or fewer CTAs when n is small.  A fixed grid above
// one wave leaves a partial second wave: at 40 registers 1184 CTAs are 1.33
// waves and the kernel streams at half the HBM rate.  Cached per kernel.
int ew_grid(const void* kernel, long long n);

template <typename... P, typename... A>
inline void ew_launch(void (*kernel)(P...), long long n, cudaStream_t st, A&&... args) {
    kernel<<<ew_grid((const void*)kernel, n), EW_THREADS, 0, st>>>(std::forward<A>(args)...);
}

inline bool valid_dims(int dim, const int* size, std::string* err, int* status) {
    if (dim < 1 || dim > 3 || !size) { *err = "dim must be 1, 2 or 3"; *status = CSIPM_ERR_INVALID; return false; }
    long long N = 1;
    for (int d = 0; d < dim; ++d) {
        if (size[d] < 2 || (size[d] % 2)) {
            *err = "every dimension must be even and >= 2";
            *status = CSIPM_ERR_ODD_DIM;
            return false;
        }
        N *= size[d];
    }
    if (N >= (1LL << 31)) { *err = "N must be below 2^31"; *status = CSIPM_ERR_UNSUPPORTED; return false; }
    return true;
}

}  // namespace csipm_internal

using namespace csipm;
using namespace csipm_internal;

// ====================================================================== handle
struct csipm_handle_s {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    csipm_options opt{};
    Geom g{};
    long long N = 0;
    double lambda = 0.0;
    FftOperator<double> op64;
    FftOperator<float> op32;        // mixed precision: the CG products
    std::string err;
    size_t bytes = 0;
    std::vector<void*> allocs;

    // reductions
    double* partials = nullptr;
    unsigned int* ticket = nullptr;
    double* slots = nullptr;        // device scalar slots
    double* hslots = nullptr;       // pinned host mirror
    CgScalars* cgs = nullptr;       // device CG scalars
    CgScalars* hcgs = nullptr;      // pinned host mirror

    // model / IPM vectors (FP64)
    double* b = nullptr;            // A^T z0
    bool sorder = false;            // solve runs in solver order (geometry.h)
    double* bs = nullptr;           // A^T z0 in solver order (when sorder)
    int4* pmap = nullptr;           // solver-order plane map (when sorder)
    double *beta = nullptr, *c = nullptr, *z1 = nullptr, *z2 = nullptr, *Qb = nullptr, *rd = nullptr;
    double *s1 = nullptr, *s2 = nullptr;    // slacks c + beta, c - beta (stored; c is output scratch)
    double *Db = nullptr, *Minv = nullptr, *rhs = nullptr, *dba = nullptr, *db = nullptr;
    double *cg_r = nullptr, *cg_p = nullptr, *cg_q = nullptr;
    // KKT plugin (allocated on first use)
    double *L1 = nullptr, *L2 = nullptr, *P11 = nullptr, *P12 = nullptr, *P22 = nullptr;
    double *k_b = nullptr, *k_x = nullptr, *k_r = nullptr, *k_p = nullptr, *k_q = nullptr;
    // Gondzio plugin (allocated on first use)
    double *gz_Dp = nullptr, *gz_Dq = nullptr, *gz_P11 = nullptr, *gz_P12 = nullptr, *gz_P22 = nullptr;
    double *gz_t1 = nullptr, *gz_t2 = nullptr;
    const double* z0 = nullptr;     // the caller's z0 (FFTParameters.z0: outlives the handle)
    // mixed precision: FP32 copies of the Schur diagonal / preconditioner and the FP32 CG vectors
    float *f_Db = nullptr, *f_Minv = nullptr, *f_r = nullptr, *f_p = nullptr, *f_q = nullptr, *f_x = nullptr;
    // FP32 Newton directions (affine, corrector) of loose mixed-precision solves
    float *f_dba = nullptr, *f_db = nullptr;
    int refinements = 0;
    // CUDA graphs of the whole CG loop (a conditional while node), one per
    // iterate vector (FP64: dba, db; FP32: f_x, f_dba, f_db), captured on first use
    cudaGraphExec_t cg_exec64[2] = {nullptr, nullptr};
    cudaGraphExec_t cg_exec32[3] = {nullptr, nullptr, nullptr};
    cudaGraphExec_t admm_exec[2] = {nullptr, nullptr};   // ADMM x-update CG, one per x buffer
    // csipm_solve's device control block (stop test, tolerances) and the
    // graph of whole interior-point iterations, captured on first use
    IpmCtl* ctl = nullptr;
    IpmCtl* hctl = nullptr;         // pinned host mirror
    cudaGraphExec_t ipm_exec = nullptr;
    int ipm_body_kernels = 0;       // kernels of one graph iteration outside its CG loops
    bool ipm_graph_off = false;     // its capture failed: csipm_solve runs plain iterations
    bool graphs_off = false;        // a capture failed: plain launches
    bool diag64_stale = false;      // FP64 Db/Minv not yet computed for this iterate (mixed precision)
    int resid_kind = 0;             // where the last Newton solve left rhs - K x (RESID_*)
    int fallbacks = 0;              // mixed Newton solves finished in FP64 after an FP32 breakdown

    // counters / timers
    int matvecs = 0;
    long long launches = 0;
    double krylov_ms = 0.0, total_ms = 0.0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t ev_rp[2] = {nullptr, nullptr};   // around each residual pass

    cudaMemPool_t pool = nullptr;   // device_pool(device): every device buffer of the handle
    static constexpr size_t HSLOT_BYTES = sizeof(double) * 64;   // SL_COUNT slots
    static constexpr size_t HCGS_BYTES = 64;                     // >= sizeof(CgScalars)
    static constexpr size_t HCTL_BYTES = 256;                    // >= sizeof(IpmCtl)
    void* hmiss = nullptr;          // pinned bounce buffer of the missing indices (csipm_create)
    size_t hmiss_bytes = 0;

    ~csipm_handle_s() {
        if (hmiss) {
            cudaStreamSynchronize(stream);   // the upload from it has completed
            pinned_put(hmiss, hmiss_bytes);
        }
        for (auto& g : cg_exec64)
            if (g) cudaGraphExecDestroy(g);
        for (auto& g : cg_exec32)
            if (g) cudaGraphExecDestroy(g);
        for (auto& g : admm_exec)
            if (g) cudaGraphExecDestroy(g);
        if (ipm_exec) cudaGraphExecDestroy(ipm_exec);
        if (hctl) pinned_put(hctl, HCTL_BYTES);
        for (void* p : allocs) cudaFreeAsync(p, stream);
        allocs.clear();
        op64.release();
        op32.release();
        if (hslots) pinned_put(hslots, HSLOT_BYTES);
        if (hcgs) pinned_put(hcgs, HCGS_BYTES);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        for (auto& e : ev_rp)
            if (e) cudaEventDestroy(e);
        if (own_stream && stream) cudaStreamDestroy(stream);
    }

    template <typename P>
    bool alloc(P** p, size_t count) {
        void* q = nullptr;
        if (cudaMallocFromPoolAsync(&q, sizeof(P) * count, pool, stream) != cudaSuccess) {
            err = "out of device memory";
            return false;
        }
        allocs.push_back(q);
        bytes += sizeof(P) * count;
        *p = reinterpret_cast<P*>(q);
        return true;
    }

    RedWorkspace ws(double* out) const { return RedWorkspace{partials, ticket, out}; }
};

namespace csipm_internal {


inline int fail(csipm_handle h, int status, const std::string& msg) {
    if (h) h->err = msg;
    set_last_error(msg);
    return status;
}

#define CK(call)                                                                        \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess)                                                          \
            return fail(h, CSIPM_ERR_CUDA, std::string("CUDA: ") + cudaGetErrorString(e_) + " at " #call); \
    } while (0)

// slot indices in h->slots
enum { SL_RED = 0, SL_MAXB = 16, SL_SS = 24, SL_DUMMY = 32, SL_DOT = 40, SL_SIGMU = 48, SL_ALPHA = 49, SL_Z0SQ = 50,
       SL_COUNT = 64 };

// ------------------------------------------------------------------ pass dispatch
// Strided pass along `axis`: the two-level register kernel when the axis has
// an instantiated factor pair and the epilogue is a hot-path one, else the
// persistent Stockham kernel.
template <typename T, bool INV, int IN, int OUT, typename TS, class Epi>
cudaError_t run_strided(FftOperator<T>& op, int axis, const PassArgs<T>& a, const TS* src, const Epi& epi,
                        cudaStream_t st) {
    if constexpr (Fft2S<T, INV, IN, OUT, TS, Epi>::value) {
        const int A = axis == 3 ? op.s3_A : op.s2_A, B = axis == 3 ? op.s3_B : op.s2_B;
        if (A) return launch_strided2<T, INV, IN, OUT, TS, Epi>(A, B, a, src, epi, st);
    }
    if constexpr (IN == IN_SGATHER || OUT == OUT_SSCATTER) {
        return cudaErrorInvalidValue;   // solver order runs on the two-level kernels only
    } else {
        return launch_strided<T, INV, IN, OUT>(axis == 3 ? op.s3_cfg : op.s2_cfg, a, src, epi, st);
    }
}

// Row pass: the two-level kernel for 2D/3D spectrum/real passes with an
// instantiated factor pair, else the Stockham kernel (also all 1D passes).
template <typename T, int IN, int OUT, bool MASK, typename TS, class Epi>
cudaError_t run_row(FftOperator<T>& op, const PassArgs<T>& a, const TS* src, const Epi& epi, cudaStream_t st) {
    if constexpr (Fft2R<T, IN, OUT, MASK>::value) {
        if (op.r_A && op.g.dim >= 2) return launch_row2<T, IN, OUT, MASK>(op.r_A, op.r_B, a, st);
    }
    return launch_row<T, IN, OUT, MASK>(op.row_cfg, a, src, epi, st);
}

// True when beta-space vectors of the solve can be kept in solver order
// (geometry.h): the gather and scatter passes along dim 2 then run on the
// two-level kernels.
template <typename T>
inline bool solver_order_ok(const FftOperator<T>& op) {
    return op.g.dim >= 2 && op.s2_A != 0;
}

// ------------------------------------------------------------------ operator
// SOL: x and the epilogue's beta-space operands are in solver order
// (requires solver_order_ok(op)).
template <typename T, typename TS, class Epi, bool SOL = false>
cudaError_t op_AtA(FftOperator<T>& op, const TS* x, const Epi& epi, const int* skip, cudaStream_t st) {
    const Geom& g = op.g;
    const double sc = 1.0 / (2.0 * (double)g.N);
    const bool mask = op.maskw != nullptr;
    EpiStore<double> none{nullptr};
    cudaError_t e;
    PassArgs<T> ra = op.row_args(sc, nullptr, nullptr);
    ra.skip = skip;
    constexpr int GIN = SOL ? IN_SGATHER : IN_GATHER;
    constexpr int SOUT = SOL ? OUT_SSCATTER : OUT_SCATTER;
    if constexpr (SOL) {
        if (!solver_order_ok(op)) return cudaErrorInvalidValue;
    } else if (g.dim == 1 && op.l1P) {
        e = l1d_first(op, x, skip, st);
        if (e != cudaSuccess) return e;
        e = mask ? l1d_row<T, IN_SPEC, OUT_SPEC, true>(op, sc, nullptr, nullptr, skip, st)
                 : l1d_row<T, IN_SPEC, OUT_SPEC, false>(op, sc, nullptr, nullptr, skip, st);
        if (e != cudaSuccess) return e;
        e = l1d_lines_forward(op, skip, st);
        if (e != cudaSuccess) return e;
        return l1d_post(op, epi, skip, st);
    } else if (g.dim == 1) {
        return mask ? run_row<T, IN_GATHER, OUT_SCATTER, true>(op, ra, x, epi, st)
                    : run_row<T, IN_GATHER, OUT_SCATTER, false>(op, ra, x, epi, st);
    }
    if (g.dim == 2) {
        PassArgs<T> a2 = op.strided_args(2);
        a2.skip = skip;
        e = run_strided<T, true, GIN, OUT_SPEC>(op, 2, a2, x, none, st);
        if (e != cudaSuccess) return e;
        e = mask ? run_row<T, IN_SPEC, OUT_SPEC, true>(op, ra, (const double*)nullptr, none, st)
                 : run_row<T, IN_SPEC, OUT_SPEC, false>(op, ra, (const double*)nullptr, none, st);
        if (e != cudaSuccess) return e;
        return run_strided<T, false, IN_SPEC, SOUT>(op, 2, a2, (const double*)nullptr, epi, st);
    }
    // 3D: the beta-side passes run along dim 2 (line stride N1/2+1 elements),
    // the plain spectrum passes along dim 3 (stride (N1/2+1)*N2)
    PassArgs<T> a3 = op.strided_args(3), a2 = op.strided_args(2);
    a3.skip = skip;
    a2.skip = skip;
    e = run_strided<T, true, GIN, OUT_SPEC>(op, 2, a2, x, none, st);
    if (e != cudaSuccess) return e;
    e = run_strided<T, true, IN_SPEC, OUT_SPEC>(op, 3, a3, (const double*)nullptr, none, st);
    if (e != cudaSuccess) return e;
    e = mask ? run_row<T, IN_SPEC, OUT_SPEC, true>(op, ra, (const double*)nullptr, none, st)
             : run_row<T, IN_SPEC, OUT_SPEC, false>(op, ra, (const double*)nullptr, none, st);
    if (e != cudaSuccess) return e;
    e = run_strided<T, false, IN_SPEC, OUT_SPEC>(op, 3, a3, (const double*)nullptr, none, st);
    if (e != cudaSuccess) return e;
    return run_strided<T, false, IN_SPEC, SOUT>(op, 2, a2, (const double*)nullptr, epi, st);
}

// x = P(sqrt(N) Re ifft(B beta))
template <typename T, typename TS>
cudaError_t op_A(FftOperator<T>& op, const TS* beta, T* x, cudaStream_t st) {
    const Geom& g = op.g;
    const bool mask = op.maskw != nullptr;
    EpiStore<double> none{nullptr};
    PassArgs<T> ra = op.row_args(1.0 / std::sqrt((double)g.N), nullptr, x);
    cudaError_t e;
    if (g.dim == 1 && op.l1P) {
        e = l1d_first(op, beta, nullptr, st);
        if (e != cudaSuccess) return e;
        return mask ? l1d_row<T, IN_SPEC, OUT_REAL, true>(op, ra.scale, nullptr, x, nullptr, st)
                    : l1d_row<T, IN_SPEC, OUT_REAL, false>(op, ra.scale, nullptr, x, nullptr, st);
    }
    if (g.dim == 1)
        return mask ? run_row<T, IN_GATHER, OUT_REAL, true>(op, ra, beta, none, st)
                    : run_row<T, IN_GATHER, OUT_REAL, false>(op, ra, beta, none, st);
    if (g.dim == 3) {
        e = run_strided<T, true, IN_GATHER, OUT_SPEC>(op, 2, op.strided_args(2), beta, none, st);
        if (e != cudaSuccess) return e;
        e = run_strided<T, true, IN_SPEC, OUT_SPEC>(op, 3, op.strided_args(3), (const double*)nullptr, none, st);
    } else {
        e = run_strided<T, true, IN_GATHER, OUT_SPEC>(op, 2, op.strided_args(2), beta, none, st);
    }
    if (e != cudaSuccess) return e;
    return mask ? run_row<T, IN_SPEC, OUT_REAL, true>(op, ra, (const double*)nullptr, none, st)
                : run_row<T, IN_SPEC, OUT_REAL, false>(op, ra, (const double*)nullptr, none, st);
}

// beta = B^T(fft(z)/sqrt(N)) through the epilogue
template <typename T, class Epi>
cudaError_t op_At(FftOperator<T>& op, const T* z, const Epi& epi, cudaStream_t st) {
    const Geom& g = op.g;
    EpiStore<double> none{nullptr};
    PassArgs<T> ra = op.row_args(1.0 / (2.0 * std::sqrt((double)g.N)), z, nullptr);
    cudaError_t e;
    if (g.dim == 1 && op.l1P) {
        e = l1d_row<T, IN_REAL, OUT_SPEC, false>(op, ra.scale, z, nullptr, nullptr, st);
        if (e != cudaSuccess) return e;
        e = l1d_lines_forward(op, nullptr, st);
        if (e != cudaSuccess) return e;
        return l1d_post(op, epi, nullptr, st);
    }
    if (g.dim == 1) return run_row<T, IN_REAL, OUT_SCATTER, false>(op, ra, (const double*)nullptr, epi, st);
    e = run_row<T, IN_REAL, OUT_SPEC, false>(op, ra, (const double*)nullptr, none, st);
    if (e != cudaSuccess) return e;
    if (g.dim == 2) return run_strided<T, false, IN_SPEC, OUT_SCATTER>(op, 2, op.strided_args(2), (const double*)nullptr, epi, st);
    e = run_strided<T, false, IN_SPEC, OUT_SPEC>(op, 3, op.strided_args(3), (const double*)nullptr, none, st);
    if (e != cudaSuccess) return e;
    return run_strided<T, false, IN_SPEC, OUT_SCATTER>(op, 2, op.strided_args(2), (const double*)nullptr, epi, st);
}

inline bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

inline int passes_per_product(const Geom& g) {
    return g.dim == 3 ? 5 : (g.dim == 2 ? 3 : (g.m1 > L1D_MIN_M ? 4 : 1));
}

inline int read_slots(csipm_handle h, int first, int count) {
    CK(cudaMemcpyAsync(h->hslots + first, h->slots + first, sizeof(double) * count, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return CSIPM_OK;
}


// A^T A for the solve's vectors (solver order when the handle uses it)
template <class Epi>
cudaError_t solve_AtA(csipm_handle h, const double* x, const Epi& epi, const int* skip, cudaStream_t st) {
    return h->sorder ? op_AtA<double, double, Epi, true>(h->op64, x, epi, skip, st)
                     : op_AtA<double, double, Epi, false>(h->op64, x, epi, skip, st);
}

template <class Epi>
cudaError_t solve_AtA32(csipm_handle h, const float* x, const Epi& epi, const int* skip, cudaStream_t st) {
    return h->sorder ? op_AtA<float, float, Epi, true>(h->op32, x, epi, skip, st)
                     : op_AtA<float, float, Epi, false>(h->op32, x, epi, skip, st);
}

// signed permutation reference order <-> solver order (n = N entries)
cudaError_t to_solver_order(const Geom& g, const double* ref, double* sol, cudaStream_t st);
cudaError_t to_reference_order(const Geom& g, const double* sol, double* ref, cudaStream_t st);

enum { RESID_NONE = 0, RESID_CG64 = 1, RESID_F32 = 2 };   // none / FP64 in cg_r / FP32 in f_r

// floor of csipm_solve's forcing term: no Newton solve is asked for more than
// FP32 products reach, so FP64 and mixed precision take the same iterates
constexpr double CG_FORCING_FLOOR = 1e-6;

// the interior-point vectors of csipm_solve / csipm_admm, allocated on first use
int ensure_ipm_buffers(csipm_handle h);

// Newton solves of the condensed system K x = rhs.  has_x0: x holds a start;
// r0v (optional, with has_x0): rhs - K x0 is already known and no product
// is spent on it.  xf (schur_mixed, optional): the start and the result are
// held in FP32 there instead of x (x is then scratch).  ready (with xf): the
// kernel that produced the right-hand side (or the warm-start residual) also
// wrote the FP32 CG start (f_r, f_p, h->cgs) for round 0.  On return
// h->resid_kind says where the residual
// rhs - K x of the result is held (RESID_*).
// rtol_dev (optional): the device copy of rtol the CG thresholds are read
// from (csipm_solve's control block: plain launches then read the same value
// graph replays do); rin_dev likewise for round 0 of a mixed solve.
int schur_cg(csipm_handle h, const double* rhs, double* x, bool has_x0, double rtol, int maxit, int* iters,
             const double* r0v = nullptr, const double* rtol_dev = nullptr);
int schur_mixed(csipm_handle h, const double* rhs, double* x, bool has_x0, double rtol, int maxit, int* iters,
                const double* r0v = nullptr, float* xf = nullptr, bool ready = false,
                const double* rin_dev = nullptr);
int ensure_kkt_buffers(csipm_handle h);
int ensure_gondzio_buffers(csipm_handle h);

}  // namespace csipm_internal
