// C ABI (include/csipm.h), part 5: batched interior-point solves.
//
// csipm_solve_batch advances many recoveries of uneven sizes together, one
// kernel launch per step for all of them.  Each recovery is an ordinary
// handle (csipm_create: its plans, twiddles, mask, spectrum, A^T z0,
// reduction workspace and control block).  The batch writes an instance
// table to device memory — per instance its vector pointers (the offsets of
// its data), size, lambda, reduction workspace, control block and the
// PassArgs of its FFT passes (run-time plans: any length) — and launches
// every element kernel and every FFT pass once with gridDim.y = instances.
// Block (x, y) works on instance y; reductions complete per instance
// (RedWorkspace::xonly); the persistent Stockham passes walk each instance's
// tiles with the same gridDim.x blocks.  An instance that has stopped
// (converged, max_iter, non-finite) returns at once from every kernel (its
// control block's status, or its CG scalars' done flag inside a CG loop).
//
// The method is csipm_solve's FP64 path — the same kernel bodies, the same
// device stop test and forcing term — in the reference packing, so each
// instance takes csipm_solve's iterates up to the order of floating-point
// sums (the FFT passes are the Stockham kernels, not the two-level ones).
// The reference has no counterpart: it solves one recovery per call
// (src/CompressedSensingIPM.jl:31-36).
#include <chrono>

#include "internal.h"

namespace csipm_internal {

// CG iterations of one lockstep loop at most (csipm_solve's graph cap)
constexpr int BATCH_CG_CAP = 2000;

// ------------------------------------------------------------------ instance table
struct BInst {
    long long n;
    double lam;
    int precond;
    int pad;
    const double* b;     // A^T z0, reference order
    double *beta, *s1, *s2, *z1, *z2, *Qb, *rd, *Db, *Minv, *rhs, *dba, *db, *r, *p, *q, *c;
    double* slots;
    double* partials;
    unsigned int* ticket;
    IpmCtl* ctl;
    CgScalars* cgs;
    __device__ __forceinline__ RedWorkspace ws(double* out) const { return RedWorkspace{partials, ticket, out, 1}; }
    __device__ __forceinline__ bool running() const { return ctl->status == IPM_RUNNING; }
};

// One FFT pass of one instance: its arguments, source and epilogue; the
// long-row fields serve the four-step 1D passes.
template <class Epi>
struct BPass {
    PassArgs<double> a;
    const double* src;
    Epi epi;
    const double2* twN;
    int P, Q, RB, TB;
};

// ------------------------------------------------------------------ element kernels
// Every wrapper reads its instance (blockIdx.y) and calls the kernel body
// csipm_solve launches; an instance that has stopped returns at once (all
// its blocks alike, so no reduction waits on it).
__global__ void __launch_bounds__(EW_THREADS) bk_init1(const BInst* __restrict__ I) {
    const BInst& q = I[blockIdx.y];
    ipm_init1_kernel_body(q.n, q.b, q.lam, q.beta, q.ws(q.slots + SL_MAXB));
}

__global__ void __launch_bounds__(EW_THREADS) bk_init2(const BInst* __restrict__ I) {
    const BInst& q = I[blockIdx.y];
    ipm_init2_kernel_body(q.n, q.b, q.Qb, q.lam, q.beta, q.slots + SL_MAXB, q.s1, q.s2, q.z1, q.z2);
}

// control blocks take ||z0||^2 and the KKT scale from the slots (one thread per instance)
__global__ void bk_ctl_start(const BInst* __restrict__ I, int count) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const BInst& q = I[k];
    q.ctl->z0sq = q.slots[SL_Z0SQ];
    q.ctl->kkt_scale = fmax(1.0, q.slots[SL_MAXB + 1]);
}

__global__ void __launch_bounds__(EW_THREADS, 3) bk_resid(const BInst* __restrict__ I, int step) {
    const BInst& q = I[blockIdx.y];
    if (!q.running()) return;
    ipm_resdiag_kernel_body<float, double>(q.n, q.b, q.Qb, q.lam, q.beta, q.s1, q.s2, q.z1, q.z2,
                                           step ? q.dba : nullptr, step ? q.db : nullptr, q.slots + SL_SIGMU,
                                           q.slots + SL_ALPHA, q.rd, q.Db, q.Minv, (float*)nullptr, (float*)nullptr,
                                           q.precond, q.rhs, q.ws(q.slots + SL_RED), (float*)nullptr,
                                           (float*)nullptr, (CgScalars*)nullptr, DevScalar());
}

// stop test per instance; a stopped instance also closes its CG scalars so
// the CG loops of the step skip it
__global__ void bk_stop(const BInst* __restrict__ I, int count) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const BInst& q = I[k];
    if (!q.running()) return;
    ipm_stop_kernel_body(q.slots + SL_RED, q.ctl, 0, 0);
    if (q.ctl->status != IPM_RUNNING) q.cgs->done = 1;
}

__global__ void __launch_bounds__(EW_THREADS) bk_zero(const BInst* __restrict__ I, int which) {
    const BInst& q = I[blockIdx.y];
    if (!q.running()) return;
    double* x = which ? q.db : q.dba;
    CSIPM_GRID_LOOP(i, q.n) x[i] = 0.0;
}

// CG start r = rhs, p = Minv r at this iteration's Newton tolerance
// (from = 0: the predictor's right-hand side; 1: the corrector's warm-start
// residual, which the corrector right-hand side pass wrote to rd)
__global__ void __launch_bounds__(EW_THREADS) bk_cg_init(const BInst* __restrict__ I, int from) {
    const BInst& q = I[blockIdx.y];
    if (!q.running()) return;
    cg_init_kernel_body<double>(q.n, from ? q.rd : q.rhs, (const double*)nullptr, 0, q.precond ? q.Minv : nullptr,
                                q.r, q.p, q.ws(q.slots + SL_DUMMY), q.cgs, 0.0, DevScalar(0.0, &q.ctl->rt));
}

__global__ void __launch_bounds__(EW_THREADS) bk_cg_update(const BInst* __restrict__ I, int it, int which) {
    const BInst& q = I[blockIdx.y];
    cg_update_kernel_body<double, double>(q.n, it, which ? q.db : q.dba, q.r, q.p, q.q, q.precond ? q.Minv : nullptr,
                                          q.ws(q.slots + SL_DUMMY), q.cgs);
}

__global__ void __launch_bounds__(EW_THREADS) bk_cg_pupdate(const BInst* __restrict__ I, int it) {
    const BInst& q = I[blockIdx.y];
    cg_pupdate_kernel_body<double>(q.n, it, q.r, q.precond ? q.Minv : nullptr, q.p, q.cgs);
}

// after a CG loop: count its iterations; a breakdown stops the instance
// (csipm_solve reports it as non-finite); one thread per instance
__global__ void bk_cg_post(const BInst* __restrict__ I, int count) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const BInst& q = I[k];
    if (!q.running()) return;
    q.ctl->cg_iter += q.cgs->iters;
    if (q.cgs->breakdown) q.ctl->status = IPM_NONFINITE;
}

// instances still iterating a CG loop (done clear) -> *out
__global__ void bk_cg_active(const BInst* __restrict__ I, int count, int* __restrict__ out) {
    __shared__ int s;
    if (threadIdx.x == 0) s = 0;
    __syncthreads();
    int c = 0;
    for (int k = threadIdx.x; k < count; k += blockDim.x) c += (I[k].running() && !I[k].cgs->done) ? 1 : 0;
    atomicAdd(&s, c);
    __syncthreads();
    if (threadIdx.x == 0) *out = s;
}

__global__ void bk_running(const BInst* __restrict__ I, int count, int* __restrict__ out) {
    __shared__ int s;
    if (threadIdx.x == 0) s = 0;
    __syncthreads();
    int c = 0;
    for (int k = threadIdx.x; k < count; k += blockDim.x) c += I[k].running() ? 1 : 0;
    atomicAdd(&s, c);
    __syncthreads();
    if (threadIdx.x == 0) *out = s;
}

__global__ void __launch_bounds__(EW_THREADS, 3) bk_stepstats(const BInst* __restrict__ I, int corrector) {
    const BInst& q = I[blockIdx.y];
    if (!q.running()) return;
    ipm_stepstats_kernel_body<double>(q.n, q.lam, q.s1, q.s2, q.z1, q.z2, corrector ? q.dba : nullptr,
                                      corrector ? q.slots + SL_SIGMU : nullptr, corrector ? q.db : q.dba,
                                      q.ws(q.slots + SL_SS));
}

__global__ void bk_sigma(const BInst* __restrict__ I, int count) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const BInst& q = I[k];
    if (!q.running()) return;
    ipm_sigma_kernel_body(q.slots + SL_SS, q.ctl, q.slots + SL_SIGMU);
}

__global__ void bk_alpha(const BInst* __restrict__ I, int count) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const BInst& q = I[k];
    if (!q.running()) return;
    ipm_alpha_kernel_body(q.slots + SL_SS, q.ctl, q.slots + SL_ALPHA);
}

// corrector right-hand side; rd receives the warm-start residual
// rhs_c - K dba = rhs_c - rhs_p + r_p (r_p: the predictor CG's residual) and
// db the warm start dba
__global__ void __launch_bounds__(EW_THREADS) bk_rhs(const BInst* __restrict__ I) {
    const BInst& q = I[blockIdx.y];
    if (!q.running()) return;
    ipm_rhs_kernel_body<double, double>(q.n, q.lam, q.s1, q.s2, q.z1, q.z2, q.rd, (const double*)q.dba,
                                        q.slots + SL_SIGMU, q.rhs, (const double*)q.r, q.db, (float*)nullptr,
                                        (float*)nullptr, (const float*)nullptr, (CgScalars*)nullptr,
                                        q.ws(q.slots + SL_DUMMY), DevScalar());
}

__global__ void __launch_bounds__(EW_THREADS) bk_beta_step(const BInst* __restrict__ I) {
    const BInst& q = I[blockIdx.y];
    if (!q.running()) return;
    ipm_beta_step_kernel_body<double>(q.n, q.beta, q.db, q.slots + SL_ALPHA);
}

// ------------------------------------------------------------------ FFT pass kernels
template <int TB, bool INV, int IN, int OUT, class Epi>
__global__ void __launch_bounds__(256) bk_strided(const BPass<Epi>* __restrict__ B) {
    const BPass<Epi>& e = B[blockIdx.y];
    strided_pass_kernel_body<double, TB, INV, IN, OUT, double, Epi>(e.a, e.src, e.epi);
}

template <int IN, int OUT, bool MASK, class Epi>
__global__ void __launch_bounds__(256) bk_row(const BPass<Epi>* __restrict__ B) {
    const BPass<Epi>& e = B[blockIdx.y];
    row_pass_kernel_body<double, IN, OUT, MASK, double, Epi>(e.a, e.src, e.epi);
}

template <class Epi>
__global__ void __launch_bounds__(256) bk_l1d_first(const BPass<Epi>* __restrict__ B) {
    const BPass<Epi>& e = B[blockIdx.y];
    l1d_first_kernel_body<double, double>(e.a, e.src, e.twN, e.P, e.Q, e.TB);
}

template <bool MASK, class Epi>
__global__ void __launch_bounds__(256) bk_l1d_row(const BPass<Epi>* __restrict__ B) {
    const BPass<Epi>& e = B[blockIdx.y];
    l1d_row_kernel_body<double, IN_SPEC, OUT_SPEC, MASK>(e.a, e.twN, e.P, e.Q, e.RB);
}

template <class Epi>
__global__ void __launch_bounds__(256) bk_l1d_post(const BPass<Epi>* __restrict__ B) {
    const BPass<Epi>& e = B[blockIdx.y];
    l1d_post_kernel_body<double, Epi>(e.a, e.twN, e.epi);
}

// ------------------------------------------------------------------ host side
// The pass sequence of one A'A product for the batch's pipeline kind, over
// tables of per-instance pass arguments (one table per pass, built once).
enum { PK_1D = 0, PK_1DL = 1, PK_2D = 2, PK_3D = 3 };

template <class Epi>
struct BProduct {
    int kind = 0;
    bool mask = false;
    int count = 0;
    // device tables, one per pass (up to 5)
    BPass<Epi>* tab[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    // launch shapes
    int tb[5] = {0, 0, 0, 0, 0};
    size_t smem[5] = {0, 0, 0, 0, 0};
    int gx[5] = {0, 0, 0, 0, 0};
    int npass = 0;
};

struct BatchState {
    int count = 0;
    cudaStream_t st = nullptr;
    cudaMemPool_t pool = nullptr;
    std::vector<void*> allocs;
    BInst* inst = nullptr;        // device table
    int* flag = nullptr;          // device counter (active CG loops / running instances)
    int* hflag = nullptr;         // pinned mirror
    BProduct<EpiStore<double>> pq;   // Qb = A'A beta
    BProduct<EpiCG<double>> pc;      // q = A'A p + Db p, p.q
    int gx_elem = 1;
    long long launches = 0;
    char* hstage = nullptr;       // pinned staging of the tables' uploads
    size_t hstage_bytes = 0, hstage_used = 0;
    ~BatchState() {
        for (void* p : allocs) cudaFreeAsync(p, st);
        if (hflag) pinned_put(hflag, 64);
        if (hstage) {
            cudaStreamSynchronize(st);   // the uploads from it have completed
            pinned_put(hstage, hstage_bytes);
        }
    }
    // host -> device copy through the pinned staging buffer (asynchronous);
    // pageable once the buffer is full
    cudaError_t upload(void* dst, const void* src, size_t bytes) {
        const size_t at = (hstage_used + 15) & ~(size_t)15;
        if (hstage && at + bytes <= hstage_bytes) {
            std::memcpy(hstage + at, src, bytes);
            hstage_used = at + bytes;
            return cudaMemcpyAsync(dst, hstage + at, bytes, cudaMemcpyHostToDevice, st);
        }
        return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st);
    }
    template <typename P>
    bool alloc(P** p, size_t count_) {
        void* q = nullptr;
        if (cudaMallocFromPoolAsync(&q, sizeof(P) * count_, pool, st) != cudaSuccess) return false;
        allocs.push_back(q);
        *p = reinterpret_cast<P*>(q);
        return true;
    }
};

int batch_kind(csipm_handle h) {
    if (h->g.dim == 3) return PK_3D;
    if (h->g.dim == 2) return PK_2D;
    return h->op64.l1P ? PK_1DL : PK_1D;
}

// Persistent-pass grid: the batch shares one wave of the kernel's CTAs
template <typename K>
int batch_grid(K kernel, int threads, size_t smem, int count, int max_tiles) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)kernel, threads, smem) != cudaSuccess ||
        per_sm < 1) {
        cudaGetLastError();
        per_sm = 1;
    }
    const int wave = std::max(1, sms) * per_sm;
    const int g = std::max(1, (wave + count - 1) / count);
    return std::max(1, std::min(g, max_tiles));
}

// Builds the pass tables of one product kind.  x: per-instance source
// vectors (beta or p); epi: per-instance epilogues; skip: per-instance flags.
template <class Epi>
int build_product(BatchState& B, BProduct<Epi>& P, const std::vector<csipm_handle>& hs, const std::vector<const double*>& x,
                  const std::vector<Epi>& epi, const std::vector<const int*>& skip) {
    const int K = (int)hs.size();
    P.count = K;
    P.kind = batch_kind(hs[0]);
    P.mask = hs[0]->op64.maskw != nullptr;
    std::vector<std::vector<BPass<Epi>>> t;
    const double C = sizeof(double2);
    auto add = [&](int pass, const PassArgs<double>& a, const double* src, const Epi& e, const double2* twN, int Pp,
                   int Qq, int RB, int TB = 0) {
        if ((int)t.size() <= pass) t.resize(pass + 1);
        BPass<Epi> bp{};
        bp.a = a;
        bp.src = src;
        bp.epi = e;
        bp.twN = twN;
        bp.P = Pp;
        bp.Q = Qq;
        bp.RB = RB;
        bp.TB = TB;
        t[pass].push_back(bp);
    };
    for (int k = 0; k < K; ++k) {
        FftOperator<double>& op = hs[k]->op64;
        const Geom& g = op.g;
        const double sc = 1.0 / (2.0 * (double)g.N);
        EpiStore<double> none{nullptr};
        (void)none;
        if (P.kind == PK_1D) {
            PassArgs<double> ra = op.row_args(sc, nullptr, nullptr);
            ra.skip = skip[k];
            add(0, ra, x[k], epi[k], nullptr, 0, 0, 0);
            P.smem[0] = std::max(P.smem[0], op.row_cfg.smem);
            P.gx[0] = std::max(P.gx[0], op.row_cfg.tiles);
        } else if (P.kind == PK_1DL) {
            PassArgs<double> a0 = l1d_args(op, false, 1.0, skip[k]);
            add(0, a0, x[k], epi[k], op.tw1, op.l1P, op.l1Q, op.l1RB, op.l1TB);
            P.smem[0] = std::max(P.smem[0], (size_t)(2 * op.l1Q * op.l1TB * C));
            P.gx[0] = std::max(P.gx[0], (op.l1P + op.l1TB - 1) / op.l1TB);
            PassArgs<double> a1 = l1d_args(op, true, sc, skip[k]);
            add(1, a1, nullptr, epi[k], op.tw1, op.l1P, op.l1Q, op.l1RB);
            P.smem[1] = std::max(P.smem[1], (size_t)(2 * op.l1P * op.l1RB * C));
            P.gx[1] = std::max(P.gx[1], (op.l1Q + op.l1RB - 1) / op.l1RB);
            PassArgs<double> a2 = l1d_args(op, false, 1.0, skip[k]);
            a2.tw_in_smem = op.q_cfg.tw_in_smem;
            a2.n_lines = op.l1P;
            a2.n_outer = 1;
            a2.so = 0;
            a2.sx = op.l1P;
            a2.jk_mode = 2;
            add(2, a2, nullptr, epi[k], op.tw1, op.l1P, op.l1Q, op.l1RB);
            P.tb[2] = P.tb[2] ? std::min(P.tb[2], op.q_cfg.tb) : op.q_cfg.tb;
            P.smem[2] = std::max(P.smem[2], op.q_cfg.smem);
            P.gx[2] = std::max(P.gx[2], op.q_cfg.tiles);
            PassArgs<double> a3 = l1d_args(op, false, 1.0, skip[k]);
            add(3, a3, nullptr, epi[k], op.tw1, op.l1P, op.l1Q, op.l1RB);
            P.gx[3] = std::max(P.gx[3], std::min(1024, (g.m1 / 2 + 1 + 255) / 256));
        } else {
            PassArgs<double> a2 = op.strided_args(2);
            a2.skip = skip[k];
            PassArgs<double> ra = op.row_args(sc, nullptr, nullptr);
            ra.skip = skip[k];
            int pass = 0;
            add(pass, a2, x[k], epi[k], nullptr, 0, 0, 0);   // gather + inverse dim 2
            P.tb[pass] = P.tb[pass] ? std::min(P.tb[pass], op.s2_cfg.tb) : op.s2_cfg.tb;
            P.gx[pass] = std::max(P.gx[pass], op.s2_cfg.tiles);
            ++pass;
            if (P.kind == PK_3D) {
                PassArgs<double> a3 = op.strided_args(3);
                a3.skip = skip[k];
                add(pass, a3, nullptr, epi[k], nullptr, 0, 0, 0);   // inverse dim 3
                P.tb[pass] = P.tb[pass] ? std::min(P.tb[pass], op.s3_cfg.tb) : op.s3_cfg.tb;
                P.gx[pass] = std::max(P.gx[pass], op.s3_cfg.tiles);
                ++pass;
            }
            add(pass, ra, nullptr, epi[k], nullptr, 0, 0, 0);   // rows
            P.smem[pass] = std::max(P.smem[pass], op.row_cfg.smem);
            P.gx[pass] = std::max(P.gx[pass], op.row_cfg.tiles);
            ++pass;
            if (P.kind == PK_3D) {
                PassArgs<double> a3 = op.strided_args(3);
                a3.skip = skip[k];
                add(pass, a3, nullptr, epi[k], nullptr, 0, 0, 0);   // forward dim 3
                P.tb[pass] = P.tb[pass] ? std::min(P.tb[pass], op.s3_cfg.tb) : op.s3_cfg.tb;
                P.gx[pass] = std::max(P.gx[pass], op.s3_cfg.tiles);
                ++pass;
            }
            add(pass, a2, nullptr, epi[k], nullptr, 0, 0, 0);   // forward dim 2 + scatter
            P.tb[pass] = P.tb[pass] ? std::min(P.tb[pass], op.s2_cfg.tb) : op.s2_cfg.tb;
            P.gx[pass] = std::max(P.gx[pass], op.s2_cfg.tiles);
        }
    }
    P.npass = (int)t.size();
    // strided passes at the batch's common lines per CTA: shared memory for
    // the largest instance at that width (data buffers + its twiddles)
    for (int pass = 0; pass < P.npass; ++pass) {
        const bool strided = (P.kind == PK_2D || P.kind == PK_3D) ? (pass != (P.kind == PK_3D ? 2 : 1))
                                                                   : (P.kind == PK_1DL && pass == 2);
        if (!strided) continue;
        size_t sm = 0;
        for (auto& e : t[pass]) {
            const size_t data = 3 * (size_t)e.a.pl.L * (size_t)C * P.tb[pass];
            sm = std::max(sm, data + (e.a.tw_in_smem ? (size_t)e.a.Ltab * (size_t)C : 0));
        }
        P.smem[pass] = sm;
    }
    for (int pass = 0; pass < P.npass; ++pass) {
        if (!B.alloc(&P.tab[pass], t[pass].size())) return CSIPM_ERR_OOM;
        if (B.upload(P.tab[pass], t[pass].data(), sizeof(BPass<Epi>) * t[pass].size()) != cudaSuccess)
            return CSIPM_ERR_CUDA;
    }
    return CSIPM_OK;
}

template <int TB, bool INV, int IN, int OUT, class Epi>
cudaError_t launch_bstrided_tb(const BProduct<Epi>& P, int pass, cudaStream_t st) {
    auto k = bk_strided<TB, INV, IN, OUT, Epi>;
    cudaError_t e = smem_optin(k, P.smem[pass]);
    if (e != cudaSuccess) return e;
    const int gx = batch_grid(k, 256, P.smem[pass], P.count, P.gx[pass]);
    k<<<dim3(gx, P.count), 256, P.smem[pass], st>>>(P.tab[pass]);
    return cudaGetLastError();
}

template <bool INV, int IN, int OUT, class Epi>
cudaError_t launch_bstrided(const BProduct<Epi>& P, int pass, cudaStream_t st) {
    switch (P.tb[pass]) {
        case 2: return launch_bstrided_tb<2, INV, IN, OUT, Epi>(P, pass, st);
        case 4: return launch_bstrided_tb<4, INV, IN, OUT, Epi>(P, pass, st);
        case 8: return launch_bstrided_tb<8, INV, IN, OUT, Epi>(P, pass, st);
        default: return cudaErrorInvalidValue;
    }
}

template <int IN, int OUT, class Epi>
cudaError_t launch_brow(const BProduct<Epi>& P, int pass, cudaStream_t st) {
    auto run = [&](auto k) -> cudaError_t {
        cudaError_t e = smem_optin(k, P.smem[pass]);
        if (e != cudaSuccess) return e;
        const int gx = batch_grid(k, 256, P.smem[pass], P.count, P.gx[pass]);
        k<<<dim3(gx, P.count), 256, P.smem[pass], st>>>(P.tab[pass]);
        return cudaGetLastError();
    };
    return P.mask ? run(bk_row<IN, OUT, true, Epi>) : run(bk_row<IN, OUT, false, Epi>);
}

// One A'A product for every instance of the batch.
template <class Epi>
cudaError_t batch_product(BatchState& B, const BProduct<Epi>& P) {
    cudaStream_t st = B.st;
    cudaError_t e = cudaSuccess;
    B.launches += P.npass;
    if (P.kind == PK_1D) return launch_brow<IN_GATHER, OUT_SCATTER, Epi>(P, 0, st);
    if (P.kind == PK_1DL) {
        {
            auto k = bk_l1d_first<Epi>;
            if ((e = smem_optin(k, P.smem[0])) != cudaSuccess) return e;
            k<<<dim3(P.gx[0], P.count), 256, P.smem[0], st>>>(P.tab[0]);
        }
        {
            auto run = [&](auto k) -> cudaError_t {
                cudaError_t e2 = smem_optin(k, P.smem[1]);
                if (e2 != cudaSuccess) return e2;
                k<<<dim3(P.gx[1], P.count), 256, P.smem[1], st>>>(P.tab[1]);
                return cudaGetLastError();
            };
            if ((e = P.mask ? run(bk_l1d_row<true, Epi>) : run(bk_l1d_row<false, Epi>)) != cudaSuccess) return e;
        }
        if ((e = launch_bstrided<false, IN_SPEC, OUT_SPEC, Epi>(P, 2, st)) != cudaSuccess) return e;
        bk_l1d_post<Epi><<<dim3(P.gx[3], P.count), 256, 0, st>>>(P.tab[3]);
        return cudaGetLastError();
    }
    int pass = 0;
    if ((e = launch_bstrided<true, IN_GATHER, OUT_SPEC, Epi>(P, pass++, st)) != cudaSuccess) return e;
    if (P.kind == PK_3D && (e = launch_bstrided<true, IN_SPEC, OUT_SPEC, Epi>(P, pass++, st)) != cudaSuccess) return e;
    if ((e = launch_brow<IN_SPEC, OUT_SPEC, Epi>(P, pass++, st)) != cudaSuccess) return e;
    if (P.kind == PK_3D && (e = launch_bstrided<false, IN_SPEC, OUT_SPEC, Epi>(P, pass++, st)) != cudaSuccess) return e;
    return launch_bstrided<false, IN_SPEC, OUT_SCATTER, Epi>(P, pass, st);
}

int read_flag(BatchState& B) {
    if (cudaMemcpyAsync(B.hflag, B.flag, sizeof(int), cudaMemcpyDeviceToHost, B.st) != cudaSuccess ||
        cudaStreamSynchronize(B.st) != cudaSuccess)
        return -1;
    return *B.hflag;
}

// One Newton solve's CG loop for every running instance, in lockstep: the
// product skips instances whose loop is done, the updates return for them.
// which: 0 predictor (iterate dba), 1 corrector (db).
int batch_cg_loop(BatchState& B, int which) {
    const dim3 ge(B.gx_elem, B.count);
    int since = 0, chunk = 2;
    for (int it = 0; it < BATCH_CG_CAP; ++it) {
        cudaError_t e = batch_product(B, B.pc);
        if (e != cudaSuccess) return fail(nullptr, CSIPM_ERR_CUDA, std::string("batch CG product: ") + cudaGetErrorString(e));
        bk_cg_update<<<ge, EW_THREADS, 0, B.st>>>(B.inst, it, which);
        bk_cg_pupdate<<<ge, EW_THREADS, 0, B.st>>>(B.inst, it);
        B.launches += 2;
        if (++since >= chunk) {
            since = 0;
            if (chunk < 8) chunk *= 2;
            bk_cg_active<<<1, 256, 0, B.st>>>(B.inst, B.count, B.flag);
            B.launches += 1;
            const int active = read_flag(B);
            if (active < 0) return fail(nullptr, CSIPM_ERR_CUDA, std::string("batch CG loop: ") + cudaGetErrorString(cudaGetLastError()));
            if (active == 0) break;
        }
    }
    bk_cg_post<<<(B.count + 127) / 128, 128, 0, B.st>>>(B.inst, B.count);
    B.launches += 1;
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? CSIPM_OK : fail(nullptr, CSIPM_ERR_CUDA, std::string("batch CG loop: ") + cudaGetErrorString(e));
}

}  // namespace csipm_internal

extern "C" {

int csipm_solve_batch(csipm_handle* hs_in, int count, double* const* beta_out, csipm_stats* stats) {
    using namespace csipm_internal;
    if (!hs_in || !beta_out || count < 1) return fail(nullptr, CSIPM_ERR_INVALID, "null argument or empty batch");
    std::vector<csipm_handle> hs(hs_in, hs_in + count);
    for (int k = 0; k < count; ++k) {
        if (!hs[k] || !beta_out[k]) return fail(nullptr, CSIPM_ERR_INVALID, "null handle or output in the batch");
        if (hs[k]->device != hs[0]->device) return fail(nullptr, CSIPM_ERR_INVALID, "the batch spans devices");
        if (batch_kind(hs[k]) != batch_kind(hs[0]) || (hs[k]->op64.maskw != nullptr) != (hs[0]->op64.maskw != nullptr))
            return fail(nullptr, CSIPM_ERR_INVALID,
                        "a batch shares the dimension count, the long-row 1D passes and the presence of missing samples");
        for (int j = 0; j < k; ++j)
            if (hs[j] == hs[k]) return fail(nullptr, CSIPM_ERR_INVALID, "a handle appears twice in the batch");
    }
    for (csipm_handle h : hs) {
        const int r = ensure_ipm_buffers(h);
        if (r) return r;
    }
    BatchState B;
    B.count = count;
    B.st = hs[0]->stream;
    B.pool = hs[0]->pool;
    cudaStream_t st = B.st;
    // the handles' own streams hand over to the batch's
    cudaEvent_t ev = nullptr;
    if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) return fail(nullptr, CSIPM_ERR_CUDA, "event");
    for (csipm_handle h : hs)
        if (h->stream != st) {
            cudaEventRecord(ev, h->stream);
            cudaStreamWaitEvent(st, ev, 0);
        }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, st);
    auto done = [&](int status) {
        cudaEventDestroy(ev);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return status;
    };
    // ---- instance table and control blocks
    std::vector<BInst> I(count);
    long long nmax = 1;
    for (int k = 0; k < count; ++k) {
        csipm_handle h = hs[k];
        BInst& q = I[k];
        q.n = h->N;
        q.lam = h->lambda;
        q.precond = h->opt.preconditioner ? 1 : 0;
        q.b = h->b;
        q.beta = h->beta; q.s1 = h->s1; q.s2 = h->s2; q.z1 = h->z1; q.z2 = h->z2; q.Qb = h->Qb; q.rd = h->rd;
        q.Db = h->Db; q.Minv = h->Minv; q.rhs = h->rhs; q.dba = h->dba; q.db = h->db;
        q.r = h->cg_r; q.p = h->cg_p; q.q = h->cg_q; q.c = h->c;
        q.slots = h->slots;
        q.partials = h->partials;
        q.ticket = h->ticket;
        q.ctl = h->ctl;
        q.cgs = h->cgs;
        nmax = std::max(nmax, h->N);
        IpmCtl& c = *h->hctl;
        std::memset(&c, 0, sizeof(IpmCtl));
        const csipm_options& o = h->opt;
        c.tol = o.tol;
        c.rt_opt = o.ipm_cg_rtol;
        c.forcing = o.ipm_cg_forcing;
        c.rt_floor = CG_FORCING_FLOOR;
        c.rin_floor = CG_FORCING_FLOOR;
        c.lam = h->lambda;
        c.two_n = 2.0 * (double)h->N;
        c.max_iter = o.max_iter;
        c.k = -1;
        c.rt_next = o.ipm_cg_rtol;
        c.rin_next = o.ipm_cg_rtol;
        c.status = IPM_RUNNING;
        if (cudaMemcpyAsync(h->ctl, h->hctl, sizeof(IpmCtl), cudaMemcpyHostToDevice, st) != cudaSuccess)
            return done(fail(nullptr, CSIPM_ERR_CUDA, "control block upload failed"));
    }
    if (!B.alloc(&B.inst, count) || !B.alloc(&B.flag, 1)) return done(fail(nullptr, CSIPM_ERR_OOM, "out of device memory"));
    B.hflag = (int*)pinned_get(64);
    if (!B.hflag) return done(fail(nullptr, CSIPM_ERR_OOM, "pinned host allocation failed"));
    {
        const size_t need = sizeof(BInst) * count + 10 * sizeof(BPass<EpiCG<double>>) * count + 16 * 12;
        size_t pb = 1 << 16;
        while (pb < need) pb <<= 1;
        if ((B.hstage = (char*)pinned_get(pb)) != nullptr) B.hstage_bytes = pb;
    }
    if (B.upload(B.inst, I.data(), sizeof(BInst) * count) != cudaSuccess)
        return done(fail(nullptr, CSIPM_ERR_CUDA, "instance table upload failed"));
    {
        int dev = 0, sms = 0, per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)bk_resid, EW_THREADS, 0);
        const long long wave = (long long)std::max(1, sms) * std::max(1, per_sm);
        B.gx_elem = (int)std::max(1LL, std::min((nmax + EW_THREADS - 1) / EW_THREADS,
                                                std::max(1LL, (wave + count - 1) / count)));
    }
    // ---- product tables: Qb = A'A beta (skips stopped instances), the CG's q = A'A p + Db p
    {
        std::vector<const double*> xb(count), xp(count);
        std::vector<EpiStore<double>> es(count);
        std::vector<EpiCG<double>> ec(count);
        std::vector<const int*> sk_ipm(count), sk_cg(count);
        for (int k = 0; k < count; ++k) {
            csipm_handle h = hs[k];
            xb[k] = h->beta;
            xp[k] = h->cg_p;
            es[k] = EpiStore<double>{h->Qb};
            RedWorkspace w{h->partials, h->ticket, &h->cgs->pq, 1};
            ec[k] = EpiCG<double>{h->cg_p, h->Db, h->cg_q, w, 0.0};
            sk_ipm[k] = &h->ctl->status;
            sk_cg[k] = &h->cgs->done;
        }
        int r = build_product(B, B.pq, hs, xb, es, sk_ipm);
        if (!r) r = build_product(B, B.pc, hs, xp, ec, sk_cg);
        if (r) return done(fail(nullptr, r, "batch pass tables failed"));
    }
    const dim3 ge(B.gx_elem, count);
    const int g1 = (count + 127) / 128;
    // ---- initial point (as csipm_solve)
    bk_init1<<<ge, EW_THREADS, 0, st>>>(B.inst);
    {
        const cudaError_t e = batch_product(B, B.pq);
        if (e != cudaSuccess) return done(fail(nullptr, CSIPM_ERR_CUDA, std::string("batch product: ") + cudaGetErrorString(e)));
    }
    bk_init2<<<ge, EW_THREADS, 0, st>>>(B.inst);
    bk_ctl_start<<<g1, 128, 0, st>>>(B.inst, count);
    B.launches += 3;
    int status = CSIPM_OK;
    bool pending = false;
    for (int iter = 0;; ++iter) {
        if (iter > 0) {
            const cudaError_t e = batch_product(B, B.pq);
            if (e != cudaSuccess) {
                status = fail(nullptr, CSIPM_ERR_CUDA, std::string("batch product: ") + cudaGetErrorString(e));
                break;
            }
        }
        bk_resid<<<ge, EW_THREADS, 0, st>>>(B.inst, pending ? 1 : 0);
        bk_stop<<<g1, 128, 0, st>>>(B.inst, count);
        bk_running<<<1, 256, 0, st>>>(B.inst, count, B.flag);
        B.launches += 3;
        const int running = read_flag(B);
        if (running < 0) { status = fail(nullptr, CSIPM_ERR_CUDA, "batch synchronisation failed"); break; }
        if (running == 0) break;
        // predictor from zero
        bk_zero<<<ge, EW_THREADS, 0, st>>>(B.inst, 0);
        bk_cg_init<<<ge, EW_THREADS, 0, st>>>(B.inst, 0);
        B.launches += 2;
        if ((status = batch_cg_loop(B, 0)) != CSIPM_OK) break;
        // centring target and corrector, warm-started at dba
        bk_stepstats<<<ge, EW_THREADS, 0, st>>>(B.inst, 0);
        bk_sigma<<<g1, 128, 0, st>>>(B.inst, count);
        bk_rhs<<<ge, EW_THREADS, 0, st>>>(B.inst);
        bk_cg_init<<<ge, EW_THREADS, 0, st>>>(B.inst, 1);
        B.launches += 4;
        if ((status = batch_cg_loop(B, 1)) != CSIPM_OK) break;
        // step
        bk_stepstats<<<ge, EW_THREADS, 0, st>>>(B.inst, 1);
        bk_alpha<<<g1, 128, 0, st>>>(B.inst, count);
        bk_beta_step<<<ge, EW_THREADS, 0, st>>>(B.inst);
        B.launches += 3;
        {
            const cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) {
                status = fail(nullptr, CSIPM_ERR_CUDA, std::string("batch launch: ") + cudaGetErrorString(e));
                break;
            }
        }
        pending = true;
    }
    // ---- results
    for (int k = 0; k < count; ++k) {
        csipm_handle h = hs[k];
        if (cudaMemcpyAsync(beta_out[k], h->beta, sizeof(double) * h->N, cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
            cudaMemcpyAsync(h->hctl, h->ctl, sizeof(IpmCtl), cudaMemcpyDeviceToHost, st) != cudaSuccess) {
            status = fail(nullptr, CSIPM_ERR_CUDA, "batch result copy failed");
            break;
        }
    }
    cudaEventRecord(e1, st);
    if (cudaEventSynchronize(e1) != cudaSuccess) return done(fail(nullptr, CSIPM_ERR_CUDA, "batch synchronisation failed"));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    int first_bad = CSIPM_OK;
    for (int k = 0; k < count; ++k) {
        csipm_handle h = hs[k];
        const IpmCtl& C = *h->hctl;
        csipm_stats S{};
        S.status = status != CSIPM_OK ? status
                   : C.status == IPM_CONVERGED ? CSIPM_OK
                   : C.status == IPM_NONFINITE ? CSIPM_ERR_NONFINITE : CSIPM_ERR_IPM_MAXITER;
        S.ipm_iter = C.k;
        S.cg_iter = C.cg_iter;
        S.matvecs = C.cg_iter + C.k + 1;
        S.gap = C.gap;
        S.obj = C.obj;
        S.lasso_obj = C.F;
        S.mu = C.mu;
        S.dual_inf = C.dual_inf;
        S.solve_ms = ms;
        S.launches = B.launches;
        if (S.status != CSIPM_OK) {
            h->err = status != CSIPM_OK                  ? std::string(get_last_error())
                     : S.status == CSIPM_ERR_NONFINITE ? "non-finite iterate or CG breakdown"
                                                        : "IPM reached max_iter before the tolerance";
            if (first_bad == CSIPM_OK) first_bad = S.status;
        }
        if (stats) stats[k] = S;
    }
    if (first_bad != CSIPM_OK && status == CSIPM_OK) {
        status = first_bad;
        set_last_error("an instance of the batch did not converge (see its csipm_stats.status)");
    }
    return done(status);
}

}  // extern "C"
