// C ABI of the library (include/csipm.h): handle management, the bit-exact
// beta <-> DFT map kernels, operator dispatch, the fused PCG drivers and the
// device-resident interior-point loop.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/csipm.h"
#include "geometry.h"
#include "operator.cuh"
#include "solver_kernels.cuh"

using namespace csipm;

namespace {

thread_local std::string g_last_error;

constexpr double SQRT2_EXACT = 1.4142135623730951;

// ------------------------------------------------------------------ map kernels
// Bit-exact beta_to_DFT (src/mapping_cpu_kernels.jl:354-738): IEEE division by
// sqrt(2), Julia's signed-zero rule for a +/- im*b (real part a +/- copysign(0,b)).
__global__ void map_b2d_kernel(Geom g, int ni, const double* __restrict__ beta, double2* __restrict__ v) {
    const long long total = (long long)ni * g.n2 * g.n3;
    CSIPM_GRID_LOOP(idx, total) {
        const int i = (int)(idx % ni);
        const long long rest = idx / ni;
        const int j = (int)(rest % g.n2), k = (int)(rest / g.n2);
        const MapEntry e = decode(g, i, j, k);
        double re, im;
        if (e.kind == KIND_VERT) {
            re = beta[e.re];
            im = 0.0;
        } else {
            const double a = beta[e.re], b = beta[e.im];
            if (e.kind == KIND_PLUS) {
                re = __ddiv_rn(__dadd_rn(a, copysign(0.0, b)), SQRT2_EXACT);
                im = __ddiv_rn(b, SQRT2_EXACT);
            } else {
                re = __ddiv_rn(__dsub_rn(a, copysign(0.0, b)), SQRT2_EXACT);
                im = __ddiv_rn(-b, SQRT2_EXACT);
            }
        }
        v[idx] = make_double2(re, im);
    }
}

// Bit-exact DFT_to_beta (src/mapping_cpu_kernels.jl:2-351): reads the half spectrum only.
__global__ void map_d2b_kernel(Geom g, const double2* __restrict__ v, double* __restrict__ beta) {
    const int ni = g.m1 + 1;
    const long long total = (long long)ni * g.n2 * g.n3;
    CSIPM_GRID_LOOP(idx, total) {
        const int i = (int)(idx % ni);
        const long long rest = idx / ni;
        const int j = (int)(rest % g.n2), k = (int)(rest / g.n2);
        const MapEntry e = decode(g, i, j, k);
        if (!e.src) continue;
        const double2 z = v[i + (long long)g.ld1 * (j + (long long)g.n2 * k)];
        if (e.kind == KIND_VERT) {
            beta[e.re] = z.x;
        } else {
            beta[e.re] = __dmul_rn(SQRT2_EXACT, z.x);
            beta[e.im] = __dmul_rn(e.kind == KIND_PLUS ? SQRT2_EXACT : -SQRT2_EXACT, z.y);
        }
    }
}

int ew_blocks(long long n) {
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

bool valid_dims(int dim, const int* size, std::string* err, int* status) {
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

}  // namespace

namespace csipm {
// lets other translation units report through csipm_last_error(NULL)
void set_last_error(const std::string& msg) { g_last_error = msg; }
}  // namespace csipm

// ====================================================================== handle
struct csipm_handle_s {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    csipm_options opt{};
    Geom g{};
    long long N = 0;
    double lambda = 0.0;
    double z0sq = 0.0;
    FftOperator<double> op64;
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
    double *beta = nullptr, *c = nullptr, *z1 = nullptr, *z2 = nullptr, *Qb = nullptr, *rd = nullptr;
    double *Db = nullptr, *Minv = nullptr, *rhs = nullptr, *dba = nullptr, *db = nullptr;
    double *cg_r = nullptr, *cg_p = nullptr, *cg_q = nullptr;
    // KKT plugin (allocated on first use)
    double *L1 = nullptr, *L2 = nullptr, *P11 = nullptr, *P12 = nullptr, *P22 = nullptr;
    double *k_b = nullptr, *k_x = nullptr, *k_r = nullptr, *k_p = nullptr, *k_q = nullptr;

    // counters / timers
    int matvecs = 0;
    long long launches = 0;
    double krylov_ms = 0.0, total_ms = 0.0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;

    ~csipm_handle_s() {
        for (void* p : allocs) cudaFree(p);
        allocs.clear();
        op64.release();
        if (hslots) cudaFreeHost(hslots);
        if (hcgs) cudaFreeHost(hcgs);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (own_stream && stream) cudaStreamDestroy(stream);
    }

    template <typename P>
    bool alloc(P** p, size_t count) {
        void* q = nullptr;
        if (cudaMalloc(&q, sizeof(P) * count) != cudaSuccess) {
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

namespace {

int fail(csipm_handle h, int status, const std::string& msg) {
    if (h) h->err = msg;
    g_last_error = msg;
    return status;
}

#define CK(call)                                                                        \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess)                                                          \
            return fail(h, CSIPM_ERR_CUDA, std::string("CUDA: ") + cudaGetErrorString(e_) + " at " #call); \
    } while (0)

// slot indices in h->slots
enum { SL_RED = 0, SL_MAXB = 16, SL_SS = 24, SL_DUMMY = 32, SL_DOT = 40, SL_COUNT = 64 };

// ------------------------------------------------------------------ operator
template <typename T, typename TS, class Epi>
cudaError_t op_AtA(FftOperator<T>& op, const TS* x, const Epi& epi, const int* skip, cudaStream_t st) {
    const Geom& g = op.g;
    const double sc = 1.0 / (2.0 * (double)g.N);
    const bool mask = op.maskw != nullptr;
    EpiStore<double> none{nullptr};
    cudaError_t e;
    PassArgs<T> ra = op.row_args(sc, nullptr, nullptr);
    ra.skip = skip;
    if (g.dim == 1) {
        return mask ? launch_row<T, IN_GATHER, OUT_SCATTER, true>(op.row_cfg, ra, x, epi, st)
                    : launch_row<T, IN_GATHER, OUT_SCATTER, false>(op.row_cfg, ra, x, epi, st);
    }
    if (g.dim == 2) {
        PassArgs<T> a2 = op.strided_args(2);
        a2.skip = skip;
        e = launch_strided<T, true, IN_GATHER, OUT_SPEC>(op.s2_cfg, a2, x, none, st);
        if (e != cudaSuccess) return e;
        e = mask ? launch_row<T, IN_SPEC, OUT_SPEC, true>(op.row_cfg, ra, (const double*)nullptr, none, st)
                 : launch_row<T, IN_SPEC, OUT_SPEC, false>(op.row_cfg, ra, (const double*)nullptr, none, st);
        if (e != cudaSuccess) return e;
        return launch_strided<T, false, IN_SPEC, OUT_SCATTER>(op.s2_cfg, a2, (const double*)nullptr, epi, st);
    }
    PassArgs<T> a3 = op.strided_args(3), a2 = op.strided_args(2);
    a3.skip = skip;
    a2.skip = skip;
    e = launch_strided<T, true, IN_GATHER, OUT_SPEC>(op.s3_cfg, a3, x, none, st);
    if (e != cudaSuccess) return e;
    e = launch_strided<T, true, IN_SPEC, OUT_SPEC>(op.s2_cfg, a2, (const double*)nullptr, none, st);
    if (e != cudaSuccess) return e;
    e = mask ? launch_row<T, IN_SPEC, OUT_SPEC, true>(op.row_cfg, ra, (const double*)nullptr, none, st)
             : launch_row<T, IN_SPEC, OUT_SPEC, false>(op.row_cfg, ra, (const double*)nullptr, none, st);
    if (e != cudaSuccess) return e;
    e = launch_strided<T, false, IN_SPEC, OUT_SPEC>(op.s2_cfg, a2, (const double*)nullptr, none, st);
    if (e != cudaSuccess) return e;
    return launch_strided<T, false, IN_SPEC, OUT_SCATTER>(op.s3_cfg, a3, (const double*)nullptr, epi, st);
}

// x = P(sqrt(N) Re ifft(B beta))
template <typename T, typename TS>
cudaError_t op_A(FftOperator<T>& op, const TS* beta, T* x, cudaStream_t st) {
    const Geom& g = op.g;
    const bool mask = op.maskw != nullptr;
    EpiStore<double> none{nullptr};
    PassArgs<T> ra = op.row_args(1.0 / std::sqrt((double)g.N), nullptr, x);
    cudaError_t e;
    if (g.dim == 1)
        return mask ? launch_row<T, IN_GATHER, OUT_REAL, true>(op.row_cfg, ra, beta, none, st)
                    : launch_row<T, IN_GATHER, OUT_REAL, false>(op.row_cfg, ra, beta, none, st);
    if (g.dim == 3) {
        e = launch_strided<T, true, IN_GATHER, OUT_SPEC>(op.s3_cfg, op.strided_args(3), beta, none, st);
        if (e != cudaSuccess) return e;
        e = launch_strided<T, true, IN_SPEC, OUT_SPEC>(op.s2_cfg, op.strided_args(2), (const double*)nullptr, none, st);
    } else {
        e = launch_strided<T, true, IN_GATHER, OUT_SPEC>(op.s2_cfg, op.strided_args(2), beta, none, st);
    }
    if (e != cudaSuccess) return e;
    return mask ? launch_row<T, IN_SPEC, OUT_REAL, true>(op.row_cfg, ra, (const double*)nullptr, none, st)
                : launch_row<T, IN_SPEC, OUT_REAL, false>(op.row_cfg, ra, (const double*)nullptr, none, st);
}

// beta = B^T(fft(z)/sqrt(N)) through the epilogue
template <typename T, class Epi>
cudaError_t op_At(FftOperator<T>& op, const T* z, const Epi& epi, cudaStream_t st) {
    const Geom& g = op.g;
    EpiStore<double> none{nullptr};
    PassArgs<T> ra = op.row_args(1.0 / (2.0 * std::sqrt((double)g.N)), z, nullptr);
    cudaError_t e;
    if (g.dim == 1) return launch_row<T, IN_REAL, OUT_SCATTER, false>(op.row_cfg, ra, (const double*)nullptr, epi, st);
    e = launch_row<T, IN_REAL, OUT_SPEC, false>(op.row_cfg, ra, (const double*)nullptr, none, st);
    if (e != cudaSuccess) return e;
    if (g.dim == 2) return launch_strided<T, false, IN_SPEC, OUT_SCATTER>(op.s2_cfg, op.strided_args(2), (const double*)nullptr, epi, st);
    e = launch_strided<T, false, IN_SPEC, OUT_SPEC>(op.s2_cfg, op.strided_args(2), (const double*)nullptr, none, st);
    if (e != cudaSuccess) return e;
    return launch_strided<T, false, IN_SPEC, OUT_SCATTER>(op.s3_cfg, op.strided_args(3), (const double*)nullptr, epi, st);
}

bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

int passes_per_product(const Geom& g) { return g.dim == 3 ? 5 : (g.dim == 2 ? 3 : 1); }

int read_slots(csipm_handle h, int first, int count) {
    CK(cudaMemcpyAsync(h->hslots + first, h->slots + first, sizeof(double) * count, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return CSIPM_OK;
}

// ------------------------------------------------------------------ Schur PCG
// Solves (A'A + Db) x = rhs with preconditioner Minv (csipm_solve's inner solve).
int schur_cg(csipm_handle h, const double* rhs, double* x, bool has_x0, double rtol, int maxit, int* iters) {
    const long long n = h->N;
    const int nb = ew_blocks(n);
    cudaStream_t st = h->stream;
    const double* Minv = h->opt.preconditioner ? h->Minv : nullptr;
    CK(cudaMemsetAsync(h->cgs, 0, sizeof(CgScalars), st));
    const int ppp = passes_per_product(h->g);
    if (has_x0) {
        EpiCG<double> ep{x, h->Db, h->cg_q, h->ws(h->slots + SL_DUMMY), 0.0};
        CK(op_AtA(h->op64, x, ep, nullptr, st));
        h->matvecs++;
        h->launches += ppp;
    } else {
        CK(cudaMemsetAsync(x, 0, sizeof(double) * n, st));
    }
    cg_init_kernel<double><<<nb, EW_THREADS, 0, st>>>(n, rhs, h->cg_q, has_x0 ? 1 : 0, Minv, h->cg_r, h->cg_p,
                                                    h->ws(h->slots + SL_DUMMY), h->cgs, 0.0, rtol);
    CK(cudaGetLastError());
    h->launches += 1;
    int chunk = 2;
    int it = 0;
    int since = 0;
    for (; it < maxit; ++it) {
        EpiCG<double> ep{h->cg_p, h->Db, h->cg_q, h->ws(&h->cgs->pq), 0.0};
        CK(op_AtA(h->op64, h->cg_p, ep, &h->cgs->done, st));
        cg_update_kernel<double, double><<<nb, EW_THREADS, 0, st>>>(n, it, x, h->cg_r, h->cg_p, h->cg_q, Minv,
                                                                    h->ws(h->slots + SL_DUMMY), h->cgs);
        cg_pupdate_kernel<double><<<nb, EW_THREADS, 0, st>>>(n, it, h->cg_r, Minv, h->cg_p, h->cgs);
        CK(cudaGetLastError());
        h->launches += ppp + 2;
        if (++since >= chunk || it + 1 == maxit) {
            since = 0;
            if (chunk < 8) chunk *= 2;
            CK(cudaMemcpyAsync(h->hcgs, h->cgs, sizeof(CgScalars), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            if (h->hcgs->done) break;
        }
    }
    CK(cudaMemcpyAsync(h->hcgs, h->cgs, sizeof(CgScalars), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    h->matvecs += h->hcgs->iters;
    *iters = h->hcgs->iters;
    if (h->hcgs->breakdown) return fail(h, CSIPM_ERR_NONFINITE, "CG breakdown (non-positive curvature or non-finite value)");
    if (!h->hcgs->done) return CSIPM_ERR_CG_MAXITER;
    return CSIPM_OK;
}

int ensure_kkt_buffers(csipm_handle h) {
    if (h->L1) return CSIPM_OK;
    const size_t n = (size_t)h->N;
    if (!h->alloc(&h->L1, n) || !h->alloc(&h->L2, n) || !h->alloc(&h->P11, n) || !h->alloc(&h->P12, n) ||
        !h->alloc(&h->P22, n) || !h->alloc(&h->k_b, 2 * n) || !h->alloc(&h->k_x, 2 * n) || !h->alloc(&h->k_r, 2 * n) ||
        !h->alloc(&h->k_p, 2 * n) || !h->alloc(&h->k_q, 2 * n))
        return fail(h, CSIPM_ERR_OOM, "out of device memory (KKT buffers)");
    return CSIPM_OK;
}

}  // namespace

// ====================================================================== C ABI
extern "C" {

int csipm_default_options(csipm_options* opt) {
    if (!opt) return CSIPM_ERR_INVALID;
    std::memset(opt, 0, sizeof(*opt));
    opt->rdft = 1;
    opt->precision = CSIPM_FP64;
    opt->preconditioner = 1;
    opt->tol = 1e-8;
    opt->max_iter = 2000;
    opt->cg_atol = 1e-12;
    opt->cg_rtol = 0.0;
    opt->cg_maxit = 0;          // 0: 2N (Krylov.jl default itmax)
    opt->ipm_cg_rtol = 1e-8;
    opt->ir_max = 3;
    opt->verbose = 0;
    opt->stream = nullptr;
    return CSIPM_OK;
}

const char* csipm_last_error(csipm_handle h) {
    return h ? h->err.c_str() : g_last_error.c_str();
}

int csipm_create(const csipm_problem* prob, const csipm_options* opt_in, csipm_handle* out) {
    csipm_handle h = nullptr;
    if (!prob || !out) return fail(h, CSIPM_ERR_INVALID, "null argument");
    *out = nullptr;
    std::string err;
    int status = 0;
    if (!valid_dims(prob->dim, prob->size, &err, &status)) return fail(h, status, err);
    if (!prob->z0) return fail(h, CSIPM_ERR_INVALID, "z0 is null");
    if (!aligned16(prob->z0)) return fail(h, CSIPM_ERR_INVALID, "z0 must be 16-byte aligned");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(h, CSIPM_ERR_NO_DEVICE, "no CUDA device");
    h = new csipm_handle_s();
    if (opt_in) h->opt = *opt_in; else csipm_default_options(&h->opt);
    if (h->opt.precision != CSIPM_FP64) {
        delete h;
        return fail(nullptr, CSIPM_ERR_UNSUPPORTED, "only CSIPM_FP64 is available in this build");
    }
    cudaGetDevice(&h->device);
    int n[3] = {prob->size[0], prob->dim >= 2 ? prob->size[1] : 1, prob->dim >= 3 ? prob->size[2] : 1};
    h->g = make_geom(prob->dim, n, n[0] / 2 + 1);
    h->N = h->g.N;
    h->lambda = prob->lambda;
    if (h->opt.cg_maxit <= 0) h->opt.cg_maxit = (int)std::min<long long>(2 * h->N, 1 << 30);
    auto bail = [&](int st, const std::string& m) { g_last_error = m; delete h; return st; };
    // NULL selects the CUDA default stream (the cuBLAS/cuFFT convention)
    h->stream = (cudaStream_t)h->opt.stream;
    h->own_stream = false;
    // mask
    std::vector<uint8_t> keep;
    if (prob->n_missing > 0) {
        if (!prob->host_missing) return bail(CSIPM_ERR_INVALID, "host_missing is null");
        keep.assign((size_t)h->N, 1u);
        for (int64_t t = 0; t < prob->n_missing; ++t) {
            const int64_t idx = prob->host_missing[t];
            if (idx < 0 || idx >= h->N) return bail(CSIPM_ERR_INVALID, "missing index out of range");
            keep[(size_t)idx] = 0u;
        }
    }
    if (!h->op64.init(h->g, keep.empty() ? nullptr : keep.data(), h->stream, &err))
        return bail(err.find("memory") != std::string::npos ? CSIPM_ERR_OOM : CSIPM_ERR_UNSUPPORTED, err);
    h->bytes += h->op64.bytes;
    // reduction workspace: enough partials for the largest grid
    size_t maxblocks = 4096;
    maxblocks = std::max<size_t>(maxblocks, (size_t)h->op64.row_cfg.grid.x);
    if (h->g.dim >= 2) maxblocks = std::max<size_t>(maxblocks, (size_t)h->op64.s2_cfg.grid.x * h->op64.s2_cfg.grid.y);
    if (h->g.dim >= 3) maxblocks = std::max<size_t>(maxblocks, (size_t)h->op64.s3_cfg.grid.x * h->op64.s3_cfg.grid.y);
    const size_t n_ = (size_t)h->N;
    if (!h->alloc(&h->partials, maxblocks * 8) || !h->alloc(&h->ticket, 1) || !h->alloc(&h->slots, SL_COUNT) ||
        !h->alloc(&h->cgs, 1) || !h->alloc(&h->b, n_) || !h->alloc(&h->beta, n_) || !h->alloc(&h->c, n_) ||
        !h->alloc(&h->z1, n_) || !h->alloc(&h->z2, n_) || !h->alloc(&h->Qb, n_) || !h->alloc(&h->rd, n_) ||
        !h->alloc(&h->Db, n_) || !h->alloc(&h->Minv, n_) || !h->alloc(&h->rhs, n_) || !h->alloc(&h->dba, n_) ||
        !h->alloc(&h->db, n_) || !h->alloc(&h->cg_r, n_) || !h->alloc(&h->cg_p, n_) || !h->alloc(&h->cg_q, n_))
        return bail(CSIPM_ERR_OOM, h->err);
    if (cudaMallocHost(&h->hslots, sizeof(double) * SL_COUNT) != cudaSuccess ||
        cudaMallocHost(&h->hcgs, sizeof(CgScalars)) != cudaSuccess)
        return bail(CSIPM_ERR_OOM, "pinned host allocation failed");
    cudaMemsetAsync(h->ticket, 0, sizeof(unsigned int), h->stream);
    cudaMemsetAsync(h->slots, 0, sizeof(double) * SL_COUNT, h->stream);
    cudaEventCreate(&h->ev0);
    cudaEventCreate(&h->ev1);
    // A^T z0 (src/fft_model.jl:60-62) and ||z0||^2
    EpiStore<double> st_b{h->b};
    {
        cudaError_t e0 = op_At(h->op64, prob->z0, st_b, h->stream);
        if (e0 != cudaSuccess) return bail(CSIPM_ERR_CUDA, std::string("A^T z0 failed: ") + cudaGetErrorString(e0));
    }
    dot2_kernel<<<ew_blocks(h->N), EW_THREADS, 0, h->stream>>>(h->N, prob->z0, prob->z0, nullptr, nullptr, h->ws(h->slots + SL_DOT));
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return bail(CSIPM_ERR_CUDA, std::string("CUDA: ") + cudaGetErrorString(e));
    if (cudaMemcpyAsync(h->hslots + SL_DOT, h->slots + SL_DOT, sizeof(double), cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
        cudaStreamSynchronize(h->stream) != cudaSuccess)
        return bail(CSIPM_ERR_CUDA, "synchronisation failed after A^T z0");
    h->z0sq = h->hslots[SL_DOT];
    *out = h;
    return CSIPM_OK;
}

int csipm_destroy(csipm_handle h) {
    if (!h) return CSIPM_ERR_INVALID;
    if (h->stream) cudaStreamSynchronize(h->stream);
    delete h;
    return CSIPM_OK;
}

int csipm_get_info(csipm_handle h, int64_t* n, size_t* device_bytes) {
    if (!h) return CSIPM_ERR_INVALID;
    if (n) *n = h->N;
    if (device_bytes) *device_bytes = h->bytes;
    return CSIPM_OK;
}

int csipm_get_Atz0(csipm_handle h, double* out) {
    if (!h || !out) return fail(h, CSIPM_ERR_INVALID, "null argument");
    CK(cudaMemcpyAsync(out, h->b, sizeof(double) * h->N, cudaMemcpyDeviceToDevice, h->stream));
    return CSIPM_OK;
}

int csipm_beta_to_dft(int dim, const int* size, int rdft, const double* beta, double* v, void* stream) {
    csipm_handle h = nullptr;
    std::string err;
    int status = 0;
    if (!valid_dims(dim, size, &err, &status)) return fail(h, status, err);
    if (!beta || !v) return fail(h, CSIPM_ERR_INVALID, "null argument");
    int n[3] = {size[0], dim >= 2 ? size[1] : 1, dim >= 3 ? size[2] : 1};
    const int ni = rdft ? n[0] / 2 + 1 : n[0];
    Geom g = make_geom(dim, n, ni);
    const long long total = (long long)ni * g.n2 * g.n3;
    map_b2d_kernel<<<ew_blocks(total), EW_THREADS, 0, (cudaStream_t)stream>>>(g, ni, beta, reinterpret_cast<double2*>(v));
    CK(cudaGetLastError());
    return CSIPM_OK;
}

int csipm_dft_to_beta(int dim, const int* size, int ld1, const double* v, double* beta, void* stream) {
    csipm_handle h = nullptr;
    std::string err;
    int status = 0;
    if (!valid_dims(dim, size, &err, &status)) return fail(h, status, err);
    if (!beta || !v) return fail(h, CSIPM_ERR_INVALID, "null argument");
    if (ld1 < size[0] / 2 + 1) return fail(h, CSIPM_ERR_INVALID, "ld1 must be >= N1/2+1");
    int n[3] = {size[0], dim >= 2 ? size[1] : 1, dim >= 3 ? size[2] : 1};
    Geom g = make_geom(dim, n, ld1);
    map_d2b_kernel<<<ew_blocks(g.Nh), EW_THREADS, 0, (cudaStream_t)stream>>>(g, reinterpret_cast<const double2*>(v), beta);
    CK(cudaGetLastError());
    return CSIPM_OK;
}

int csipm_apply_A(csipm_handle h, const double* beta, double* x) {
    if (!h || !beta || !x) return fail(h, CSIPM_ERR_INVALID, "null argument");
    if (!aligned16(x)) return fail(h, CSIPM_ERR_INVALID, "x must be 16-byte aligned");
    CK(op_A(h->op64, beta, x, h->stream));
    return CSIPM_OK;
}

int csipm_apply_At(csipm_handle h, const double* z, double* beta) {
    if (!h || !z || !beta) return fail(h, CSIPM_ERR_INVALID, "null argument");
    if (!aligned16(z)) return fail(h, CSIPM_ERR_INVALID, "z must be 16-byte aligned");
    EpiStore<double> ep{beta};
    CK(op_At(h->op64, z, ep, h->stream));
    return CSIPM_OK;
}

int csipm_apply_AtA(csipm_handle h, const double* x, double* y) {
    if (!h || !x || !y) return fail(h, CSIPM_ERR_INVALID, "null argument");
    EpiStore<double> ep{y};
    CK(op_AtA(h->op64, x, ep, nullptr, h->stream));
    h->matvecs++;
    return CSIPM_OK;
}

int csipm_obj(csipm_handle h, const double* x, double* f) {
    if (!h || !x || !f) return fail(h, CSIPM_ERR_INVALID, "null argument");
    // 1/2 ||A beta||^2 = 1/2 beta' A'A beta (P is a projection); - beta'A^T z0 ; + lambda sum(c)
    EpiStore<double> ep{h->Qb};
    CK(op_AtA(h->op64, x, ep, nullptr, h->stream));
    h->matvecs++;
    const long long n = h->N;
    dot2_kernel<<<ew_blocks(n), EW_THREADS, 0, h->stream>>>(n, x, h->Qb, x, h->b, h->ws(h->slots + SL_DOT));
    CK(cudaGetLastError());
    // sum(c) = c . 1 : reuse Minv as a ones vector would cost a fill; use a dedicated reduction
    fill_kernel<<<ew_blocks(n), EW_THREADS, 0, h->stream>>>(n, 1.0, h->rhs);
    dot2_kernel<<<ew_blocks(n), EW_THREADS, 0, h->stream>>>(n, x + n, h->rhs, nullptr, nullptr, h->ws(h->slots + SL_DOT + 2));
    CK(cudaGetLastError());
    int r = read_slots(h, SL_DOT, 3);
    if (r) return r;
    *f = 0.5 * h->hslots[SL_DOT] - h->hslots[SL_DOT + 1] + h->lambda * h->hslots[SL_DOT + 2];
    return CSIPM_OK;
}

int csipm_grad(csipm_handle h, const double* x, double* g) {
    if (!h || !x || !g) return fail(h, CSIPM_ERR_INVALID, "null argument");
    EpiGrad ep{h->b, g};
    CK(op_AtA(h->op64, x, ep, nullptr, h->stream));
    h->matvecs++;
    fill_kernel<<<ew_blocks(h->N), EW_THREADS, 0, h->stream>>>(h->N, h->lambda, g + h->N);
    CK(cudaGetLastError());
    return CSIPM_OK;
}

int csipm_cons(csipm_handle h, const double* x, double* c) {
    if (!h || !x || !c) return fail(h, CSIPM_ERR_INVALID, "null argument");
    cons_kernel<<<ew_blocks(h->N), EW_THREADS, 0, h->stream>>>(h->N, x, c);
    CK(cudaGetLastError());
    return CSIPM_OK;
}

int csipm_hprod(csipm_handle h, const double* v, double* hv, double obj_weight) {
    if (!h || !v || !hv) return fail(h, CSIPM_ERR_INVALID, "null argument");
    EpiScale ep{obj_weight, hv};
    CK(op_AtA(h->op64, v, ep, nullptr, h->stream));
    h->matvecs++;
    fill_kernel<<<ew_blocks(h->N), EW_THREADS, 0, h->stream>>>(h->N, 0.0, hv + h->N);
    CK(cudaGetLastError());
    return CSIPM_OK;
}

int csipm_kkt_build(csipm_handle h, const double* pr_diag) {
    if (!h || !pr_diag) return fail(h, CSIPM_ERR_INVALID, "null argument");
    int r = ensure_kkt_buffers(h);
    if (r) return r;
    kkt_build_kernel<<<ew_blocks(h->N), EW_THREADS, 0, h->stream>>>(h->N, pr_diag, h->L1, h->L2, h->P11, h->P12, h->P22);
    CK(cudaGetLastError());
    return CSIPM_OK;
}

int csipm_condensed_mul(csipm_handle h, double* y, const double* x, double alpha, double beta) {
    if (!h || !x || !y) return fail(h, CSIPM_ERR_INVALID, "null argument");
    if (!h->L1) return fail(h, CSIPM_ERR_INVALID, "csipm_kkt_build must be called first");
    EpiCondensed ep{x, y, h->L1, h->L2, h->N, alpha, beta};
    CK(op_AtA(h->op64, x, ep, nullptr, h->stream));
    h->matvecs++;
    return CSIPM_OK;
}

int csipm_precond_mul(csipm_handle h, double* y, const double* x, double alpha, double beta) {
    if (!h || !x || !y) return fail(h, CSIPM_ERR_INVALID, "null argument");
    if (!h->L1) return fail(h, CSIPM_ERR_INVALID, "csipm_kkt_build must be called first");
    precond_mul_kernel<<<ew_blocks(h->N), EW_THREADS, 0, h->stream>>>(h->N, y, x, h->P11, h->P12, h->P22, alpha, beta);
    CK(cudaGetLastError());
    return CSIPM_OK;
}

int csipm_kkt_mul(csipm_handle h, double* y, const double* x, double alpha, double beta) {
    if (!h || !x || !y) return fail(h, CSIPM_ERR_INVALID, "null argument");
    EpiKKT ep{x, y, h->N, alpha, beta};
    CK(op_AtA(h->op64, x, ep, nullptr, h->stream));
    h->matvecs++;
    return CSIPM_OK;
}

int csipm_jtprod(csipm_handle h, double* y, const double* x) {
    if (!h || !x || !y) return fail(h, CSIPM_ERR_INVALID, "null argument");
    jtprod_kernel<<<ew_blocks(h->N), EW_THREADS, 0, h->stream>>>(h->N, y, x);
    CK(cudaGetLastError());
    return CSIPM_OK;
}

int csipm_kkt_solve(csipm_handle h, double* w, const double* pr_diag, int* cg_iters) {
    if (!h || !w || !pr_diag) return fail(h, CSIPM_ERR_INVALID, "null argument");
    if (!h->L1) return fail(h, CSIPM_ERR_INVALID, "csipm_kkt_build must be called first");
    const long long n = h->N;
    const int nb = ew_blocks(n);
    cudaStream_t st = h->stream;
    const bool pc = h->opt.preconditioner != 0;
    const double *P11 = pc ? h->P11 : nullptr, *P12 = pc ? h->P12 : nullptr, *P22 = pc ? h->P22 : nullptr;
    cudaEventRecord(h->ev0, st);
    kkt_rhs_kernel<<<nb, EW_THREADS, 0, st>>>(n, w, pr_diag, h->k_b);
    CK(cudaMemsetAsync(h->cgs, 0, sizeof(CgScalars), st));
    kcg_init_kernel<<<nb, EW_THREADS, 0, st>>>(n, h->k_b, h->k_x, h->k_r, h->k_p, P11, P12, P22,
                                              h->ws(h->slots + SL_DUMMY), h->cgs, h->opt.cg_atol, h->opt.cg_rtol);
    CK(cudaGetLastError());
    int chunk = 2, since = 0;
    const int maxit = h->opt.cg_maxit;
    for (int it = 0; it < maxit; ++it) {
        EpiKcg ep{h->k_p, h->k_q, h->L1, h->L2, n, h->ws(&h->cgs->pq), 0.0};
        CK(op_AtA(h->op64, h->k_p, ep, &h->cgs->done, st));
        kcg_update_kernel<<<nb, EW_THREADS, 0, st>>>(n, it, h->k_x, h->k_r, h->k_p, h->k_q, P11, P12, P22,
                                                     h->ws(h->slots + SL_DUMMY), h->cgs);
        kcg_pupdate_kernel<<<nb, EW_THREADS, 0, st>>>(n, it, h->k_r, h->k_p, P11, P12, P22, h->cgs);
        CK(cudaGetLastError());
        if (++since >= chunk || it + 1 == maxit) {
            since = 0;
            if (chunk < 8) chunk *= 2;
            CK(cudaMemcpyAsync(h->hcgs, h->cgs, sizeof(CgScalars), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            if (h->hcgs->done) break;
        }
    }
    CK(cudaMemcpyAsync(h->hcgs, h->cgs, sizeof(CgScalars), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    h->matvecs += h->hcgs->iters;
    kkt_back_kernel<<<nb, EW_THREADS, 0, st>>>(n, w, h->k_x, pr_diag);
    CK(cudaGetLastError());
    cudaEventRecord(h->ev1, st);
    CK(cudaEventSynchronize(h->ev1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    h->krylov_ms += ms;
    if (cg_iters) *cg_iters = h->hcgs->iters;
    if (h->hcgs->breakdown) return fail(h, CSIPM_ERR_NONFINITE, "CG breakdown in solve_kkt");
    return CSIPM_OK;
}

int csipm_solve(csipm_handle h, double* beta_out, double* c_out, csipm_stats* stats) {
    if (!h || !beta_out) return fail(h, CSIPM_ERR_INVALID, "null argument");
    const long long n = h->N;
    const int nb = ew_blocks(n);
    cudaStream_t st = h->stream;
    const double lam = h->lambda;
    const csipm_options& o = h->opt;
    csipm_stats S{};
    const int mv0 = h->matvecs;
    const long long la0 = h->launches;
    const int ppp = passes_per_product(h->g);
    cudaEventRecord(h->ev0, st);
    // ---- initial point: beta = soft(A^T z0, lambda), z from the clipped gradient, c balanced
    ipm_init1_kernel<<<nb, EW_THREADS, 0, st>>>(n, h->b, lam, h->beta, h->ws(h->slots + SL_MAXB));
    CK(cudaGetLastError());
    {
        EpiStore<double> ep{h->Qb};
        CK(op_AtA(h->op64, h->beta, ep, nullptr, st));
        h->matvecs++;
    }
    h->launches += 2 + ppp;
    ipm_init2_kernel<<<nb, EW_THREADS, 0, st>>>(n, h->b, h->Qb, lam, h->beta, h->slots + SL_MAXB, h->c, h->z1, h->z2);
    CK(cudaGetLastError());
    {
        int r0 = read_slots(h, SL_MAXB, 2);
        if (r0) return r0;
    }
    const double kkt_scale = std::max(1.0, h->hslots[SL_MAXB + 1]);
    int status = CSIPM_ERR_IPM_MAXITER;
    double mu = 0.0, gap = 1.0;
    int k = 0;
    for (;; ++k) {
        if (k > 0) {
            EpiStore<double> ep{h->Qb};
            CK(op_AtA(h->op64, h->beta, ep, nullptr, st));
            h->matvecs++;
            h->launches += ppp;
        }
        h->launches += 1;   // residual
        ipm_residual_kernel<<<nb, EW_THREADS, 0, st>>>(n, h->b, h->Qb, lam, h->beta, h->c, h->z1, h->z2, h->rd,
                                                       h->ws(h->slots + SL_RED));
        CK(cudaGetLastError());
        int r = read_slots(h, SL_RED, RR_N);
        if (r) return r;
        const double* R = h->hslots + SL_RED;
        mu = R[RR_SZ] / (2.0 * (double)n);
        const double usq = h->z0sq - 2.0 * R[RR_BB] + R[RR_BQB];
        const double F = 0.5 * usq + lam * R[RR_L1];
        const double th = R[RR_GINF] > 0.0 ? std::min(1.0, lam / R[RR_GINF]) : 1.0;
        const double D = th * (h->z0sq - R[RR_BB]) - 0.5 * th * th * usq;
        gap = (F - D) / std::max(std::fabs(F), 1e-300);
        // scaled KKT error: the criterion that still applies when lambda = 0
        // makes the LASSO dual bound degenerate
        const double kkt = std::max(std::max(R[RR_RDINF], R[RR_RCINF]), mu) / kkt_scale;
        S.obj = 0.5 * R[RR_BQB] - R[RR_BB] + lam * R[RR_SUMC];
        S.lasso_obj = F;
        S.dual_inf = R[RR_RDINF];
        S.mu = mu;
        S.gap = gap;
        if (!std::isfinite(mu) || !std::isfinite(gap)) { status = fail(h, CSIPM_ERR_NONFINITE, "non-finite iterate"); break; }
        if (o.verbose)
            std::fprintf(stderr, "csipm it %3d  mu %.3e  gap %.3e  |rd| %.2e  |rc| %.2e  obj %.12e  cg %d\n", k, mu, gap,
                         R[RR_RDINF], R[RR_RCINF], F, S.cg_iter);
        if (gap <= o.tol || kkt <= o.tol) { status = CSIPM_OK; break; }
        if (k >= o.max_iter) { status = CSIPM_ERR_IPM_MAXITER; break; }
        ipm_diag_kernel<double><<<nb, EW_THREADS, 0, st>>>(n, h->beta, h->c, h->z1, h->z2, h->Db, h->Minv,
                                                           (double*)nullptr, (double*)nullptr, o.preconditioner);
        // ---- predictor (affine scaling)
        ipm_rhs_kernel<<<nb, EW_THREADS, 0, st>>>(n, lam, h->beta, h->c, h->z1, h->z2, h->rd, nullptr, 0.0, h->rhs);
        CK(cudaGetLastError());
        int its = 0;
        int cs = schur_cg(h, h->rhs, h->dba, false, o.ipm_cg_rtol, o.cg_maxit, &its);
        S.cg_iter += its;
        if (cs != CSIPM_OK && cs != CSIPM_ERR_CG_MAXITER) { status = cs; break; }
        ipm_stepstats_kernel<<<nb, EW_THREADS, 0, st>>>(n, lam, h->beta, h->c, h->z1, h->z2, nullptr, 0.0, h->dba,
                                                        h->ws(h->slots + SL_SS));
        CK(cudaGetLastError());
        r = read_slots(h, SL_SS, SS_N);
        if (r) return r;
        const double* Q = h->hslots + SL_SS;
        double a = std::min(1.0, std::min(Q[SS_MINP], Q[SS_MIND]));
        const double mu_aff = (Q[SS_SZ] + a * Q[SS_CROSS] + a * a * Q[SS_DD]) / (2.0 * (double)n);
        const double sigma = std::pow(std::max(mu_aff, 0.0) / mu, 3.0);
        const double sigmu = sigma * mu;
        // ---- corrector
        ipm_rhs_kernel<<<nb, EW_THREADS, 0, st>>>(n, lam, h->beta, h->c, h->z1, h->z2, h->rd, h->dba, sigmu, h->rhs);
        CK(cudaMemcpyAsync(h->db, h->dba, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
        cs = schur_cg(h, h->rhs, h->db, true, o.ipm_cg_rtol, o.cg_maxit, &its);
        S.cg_iter += its;
        if (cs != CSIPM_OK && cs != CSIPM_ERR_CG_MAXITER) { status = cs; break; }
        ipm_stepstats_kernel<<<nb, EW_THREADS, 0, st>>>(n, lam, h->beta, h->c, h->z1, h->z2, h->dba, sigmu, h->db,
                                                        h->ws(h->slots + SL_SS));
        CK(cudaGetLastError());
        r = read_slots(h, SL_SS, SS_N);
        if (r) return r;
        const double eta = std::max(0.99, 1.0 - mu);
        const double ap = std::min(1.0, eta * Q[SS_MINP]);
        const double ad = std::min(1.0, eta * Q[SS_MIND]);
        a = std::min(ap, ad);
        ipm_update_kernel<<<nb, EW_THREADS, 0, st>>>(n, lam, h->beta, h->c, h->z1, h->z2, h->dba, sigmu, h->db, a, a);
        CK(cudaGetLastError());
        h->launches += 7;   // diag, 2 rhs, 2 step statistics, update (+ CG launches counted in schur_cg)
    }
    CK(cudaMemcpyAsync(beta_out, h->beta, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    if (c_out) CK(cudaMemcpyAsync(c_out, h->c, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    cudaEventRecord(h->ev1, st);
    CK(cudaEventSynchronize(h->ev1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    S.solve_ms = ms;
    S.status = status;
    S.ipm_iter = k;
    S.matvecs = h->matvecs - mv0;
    S.launches = h->launches - la0;
    if (stats) *stats = S;
    if (status == CSIPM_ERR_IPM_MAXITER) fail(h, status, "IPM reached max_iter before the tolerance");
    return status;
}

int csipm_profile_passes(csipm_handle h, const double* x, int reps, double* ms_out, double* bytes_out,
                         char* name_out, int* npass) {
    if (!h || !x || !ms_out || !bytes_out || !npass || reps < 1) return fail(h, CSIPM_ERR_INVALID, "bad argument");
    FftOperator<double>& op = h->op64;
    const Geom& g = h->g;
    cudaStream_t st = h->stream;
    const double N = (double)g.N, Nh = (double)g.Nh;
    const double w = 8.0, cw = 16.0, maskb = op.maskw ? N / 8.0 : 0.0;
    CK(cudaMemsetAsync(h->Db, 0, sizeof(double) * g.N, st));
    EpiStore<double> none{nullptr};
    EpiCG<double> ecg{x, h->Db, h->cg_q, h->ws(h->slots + SL_DUMMY), 0.0};
    const bool mask = op.maskw != nullptr;
    PassArgs<double> ra = op.row_args(1.0 / (2.0 * N), nullptr, nullptr);
    int np = 0;
    const char* names[8];
    auto timeit = [&](auto&& launch, double bytes, const char* name) -> int {
        CK(launch());   // warm
        CK(cudaEventRecord(h->ev0, st));
        for (int r = 0; r < reps; ++r) CK(launch());
        CK(cudaEventRecord(h->ev1, st));
        CK(cudaEventSynchronize(h->ev1));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, h->ev0, h->ev1);
        ms_out[np] = ms / reps;
        bytes_out[np] = bytes;
        names[np] = name;
        ++np;
        return CSIPM_OK;
    };
    int r = 0;
    if (g.dim == 1) {
        r = timeit([&] { return mask ? launch_row<double, IN_GATHER, OUT_SCATTER, true>(op.row_cfg, ra, x, ecg, st)
                                     : launch_row<double, IN_GATHER, OUT_SCATTER, false>(op.row_cfg, ra, x, ecg, st); },
                   4 * w * N + maskb, "row: gather+C2R+mask+R2C+scatter+CG");
        if (r) return r;
    } else {
        const int ax = g.dim;   // outermost axis
        PassArgs<double> ao = op.strided_args(ax);
        const PassCfg& co = ax == 3 ? op.s3_cfg : op.s2_cfg;
        r = timeit([&] { return launch_strided<double, true, IN_GATHER, OUT_SPEC>(co, ao, x, none, st); },
                   w * N + cw * Nh, ax == 3 ? "gather+inverse dim3" : "gather+inverse dim2");
        if (r) return r;
        if (g.dim == 3) {
            PassArgs<double> a2 = op.strided_args(2);
            r = timeit([&] { return launch_strided<double, true, IN_SPEC, OUT_SPEC>(op.s2_cfg, a2, (const double*)nullptr, none, st); },
                       2 * cw * Nh, "inverse dim2");
            if (r) return r;
        }
        r = timeit([&] { return mask ? launch_row<double, IN_SPEC, OUT_SPEC, true>(op.row_cfg, ra, (const double*)nullptr, none, st)
                                     : launch_row<double, IN_SPEC, OUT_SPEC, false>(op.row_cfg, ra, (const double*)nullptr, none, st); },
                   2 * cw * Nh + maskb, "row: C2R+mask+R2C dim1");
        if (r) return r;
        if (g.dim == 3) {
            PassArgs<double> a2 = op.strided_args(2);
            r = timeit([&] { return launch_strided<double, false, IN_SPEC, OUT_SPEC>(op.s2_cfg, a2, (const double*)nullptr, none, st); },
                       2 * cw * Nh, "forward dim2");
            if (r) return r;
        }
        r = timeit([&] { return launch_strided<double, false, IN_SPEC, OUT_SCATTER>(co, ao, (const double*)nullptr, ecg, st); },
                   cw * Nh + 3 * w * N, ax == 3 ? "forward dim3+scatter+CG" : "forward dim2+scatter+CG");
        if (r) return r;
    }
    *npass = np;
    if (name_out)
        for (int k = 0; k < np; ++k) {
            std::strncpy(name_out + 32 * k, names[k], 31);
            name_out[32 * k + 31] = 0;
        }
    return CSIPM_OK;
}

int csipm_get_timers(csipm_handle h, double* operator_ms, double* elementwise_ms, double* krylov_ms, int reset) {
    if (!h) return CSIPM_ERR_INVALID;
    if (operator_ms) *operator_ms = 0.0;
    if (elementwise_ms) *elementwise_ms = 0.0;
    if (krylov_ms) *krylov_ms = h->krylov_ms;
    if (reset) h->krylov_ms = 0.0;
    return CSIPM_OK;
}

}  // extern "C"
