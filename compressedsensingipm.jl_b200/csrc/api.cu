// C ABI (include/csipm.h), part 1: handle lifecycle, the operator entry
// points, the fused Schur-complement PCG and the device-resident
// interior-point loop.  The NLPModels / KKT-plugin entry points are in
// plugin.cu, the bit-exact maps in maps.cu.
#include <limits>
#include <mutex>

#include "internal.h"
#include "tune.cuh"

namespace {
thread_local std::string g_last_error;
}  // namespace

namespace csipm {
// lets every translation unit report through csipm_last_error(NULL)
void set_last_error(const std::string& msg) { g_last_error = msg; }
const char* get_last_error() { return g_last_error.c_str(); }

namespace {
std::mutex g_pool_mu;
std::map<int, cudaMemPool_t> g_pools;
std::mutex g_pin_mu;
std::map<size_t, std::vector<void*>> g_pinned;
}  // namespace

cudaMemPool_t device_pool(int dev) {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    auto it = g_pools.find(dev);
    if (it != g_pools.end()) return it->second;
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) return nullptr;
    uint64_t keep = UINT64_MAX;   // keep freed blocks for the next handle
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    g_pools[dev] = pool;
    return pool;
}

void* pinned_get(size_t bytes) {
    {
        std::lock_guard<std::mutex> lk(g_pin_mu);
        auto& v = g_pinned[bytes];
        if (!v.empty()) {
            void* p = v.back();
            v.pop_back();
            return p;
        }
    }
    void* p = nullptr;
    if (cudaMallocHost(&p, bytes) != cudaSuccess) return nullptr;
    return p;
}

void pinned_put(void* p, size_t bytes) {
    std::lock_guard<std::mutex> lk(g_pin_mu);
    g_pinned[bytes].push_back(p);
}
}  // namespace csipm

namespace csipm_internal {

// ------------------------------------------------------------------ solver order
// One thread per solver-order pair (NI of them) and per tail entry; every
// reference index is read or written exactly once (the packing is a bijection
// between beta entries and the sources of the half spectrum).
template <bool TO_SOL>
static __global__ void solver_order_kernel(Geom g, const double* __restrict__ in, double* __restrict__ out) {
    const int64_t tail = g.N - 2 * g.NI;
    const int64_t total = g.NI + tail;
    const int pl = g.m1 - 1;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total; idx += (int64_t)gridDim.x * blockDim.x) {
        if (idx < g.NI) {
            const int i = (int)(idx % pl) + 1;
            const int64_t r = idx / pl;
            const int j = (int)(r % g.n2), k = (int)(r / g.n2);
            const MapEntry e = decode_interior(g, i, j, k);
            const double sg = e.kind == KIND_MINUS ? -1.0 : 1.0;
            if (TO_SOL) {
                reinterpret_cast<double2*>(out)[idx] = make_double2(in[e.re], sg * in[e.im]);
            } else {
                const double2 v = reinterpret_cast<const double2*>(in)[idx];
                out[e.re] = v.x;
                out[e.im] = sg * v.y;
            }
        } else {
            const int64_t t = idx - g.NI;
            const int64_t ref = sol_tail_ref(g, t);
            if (TO_SOL) out[2 * g.NI + t] = in[ref];
            else out[ref] = in[2 * g.NI + t];
        }
    }
}

// Solver-order plane map: (re, im, kind, src) of the planes i = 0 and i = M1,
// entry (p*N3 + k)*N2 + j, with re / im as solver-order tail indices.
static __global__ void plane_map_kernel(Geom g, int4* __restrict__ pm) {
    const int64_t per = (int64_t)g.n2 * g.n3;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < 2 * per;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int p = (int)(idx / per);
        const int64_t r = idx - p * per;
        const int k = (int)(r / g.n2), j = (int)(r % g.n2);
        const MapEntry e = decode(g, p ? g.m1 : 0, j, k);
        pm[idx] = make_int4((int)sol_tail(g, e.re), e.kind == KIND_VERT ? -1 : (int)sol_tail(g, e.im), e.kind, e.src);
    }
}

cudaError_t to_solver_order(const Geom& g, const double* ref, double* sol, cudaStream_t st) {
    solver_order_kernel<true><<<ew_blocks(g.N / 2 + 1), EW_THREADS, 0, st>>>(g, ref, sol);
    return cudaGetLastError();
}

cudaError_t to_reference_order(const Geom& g, const double* sol, double* ref, cudaStream_t st) {
    solver_order_kernel<false><<<ew_blocks(g.N / 2 + 1), EW_THREADS, 0, st>>>(g, sol, ref);
    return cudaGetLastError();
}

// ------------------------------------------------------------------ CG iteration loop
// Runs PCG iterations (iteration(stream, it) launches one; `it` only selects
// the parity of the double-buffered scalars) until the device `done` flag is
// set or maxit is reached.
//
// With CUDA graphs (the default) the whole loop is one graph launch: a
// conditional WHILE node whose body is two iterations followed by a
// one-thread kernel that keeps the loop going while `done` is clear and
// fewer than CG_WHILE_CAP iterations ran (the bound keeps every device loop
// finite); the graph is captured once per handle and solution vector.  The
// host reads the scalars once at the end and finishes with plain launches
// in the rare case the cap was reached.  Without graphs the flag is read
// back after 2, 4, then every 8 iterations.
constexpr int CG_WHILE_CAP = 2000;

static __global__ void cg_continue_kernel(cudaGraphConditionalHandle hnd, const CgScalars* __restrict__ sc, int cap) {
    cudaGraphSetConditional(hnd, (sc->done == 0 && sc->iters < cap) ? 1u : 0u);
}

template <class Iter>
bool build_cg_while(csipm_handle h, cudaGraphExec_t* exec, int cap, Iter& iteration) {
    cudaGraph_t graph = nullptr;
    cudaStream_t cs = nullptr;
    bool ok = cudaGraphCreate(&graph, 0) == cudaSuccess;
    cudaGraphConditionalHandle hnd = 0;
    if (ok) ok = cudaGraphConditionalHandleCreate(&hnd, graph, 1, cudaGraphCondAssignDefault) == cudaSuccess;
    cudaGraphNodeParams cp = {};
    cudaGraphNode_t node = nullptr;
    if (ok) {
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = hnd;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        ok = cudaGraphAddNode(&node, graph, nullptr, 0, &cp) == cudaSuccess;
    }
    if (ok) ok = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) == cudaSuccess;
    if (ok) {
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        ok = cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) ==
             cudaSuccess;
        if (ok) {
            ok = iteration(cs, 0) == cudaSuccess && iteration(cs, 1) == cudaSuccess;
            cg_continue_kernel<<<1, 1, 0, cs>>>(hnd, h->cgs, cap);
            ok = cudaGetLastError() == cudaSuccess && ok;
            cudaGraph_t out = nullptr;
            ok = cudaStreamEndCapture(cs, &out) == cudaSuccess && ok;
        }
    }
    if (ok) ok = cudaGraphInstantiate(exec, graph, 0) == cudaSuccess;
    if (cs) cudaStreamDestroy(cs);
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    if (!ok) *exec = nullptr;
    return ok;
}

template <class Iter>
int cg_iterations(csipm_handle h, cudaGraphExec_t* exec, int maxit, Iter&& iteration, int per_iter) {
    cudaStream_t st = h->stream;
    int it = 0;
    if (exec && h->opt.cuda_graphs && !h->graphs_off && maxit >= 2) {
        if (!*exec && !build_cg_while(h, exec, std::min(maxit, CG_WHILE_CAP), iteration)) h->graphs_off = true;
        if (*exec) {
            CK(cudaGraphLaunch(*exec, st));
            CK(cudaMemcpyAsync(h->hcgs, h->cgs, sizeof(CgScalars), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            h->launches += (long long)h->hcgs->iters * per_iter + 1;
            if (h->hcgs->done) return CSIPM_OK;
            it = h->hcgs->iters;   // cap reached (even): continue with plain launches
        }
    }
    int chunk = 2, since = 0;
    while (it < maxit) {
        CK(iteration(st, it));
        h->launches += per_iter;
        ++it;
        if (++since >= chunk || it >= maxit) {
            since = 0;
            if (chunk < 8) chunk *= 2;
            CK(cudaMemcpyAsync(h->hcgs, h->cgs, sizeof(CgScalars), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            if (h->hcgs->done) break;
        }
    }
    return CSIPM_OK;
}

// ------------------------------------------------------------------ Schur PCG
// Solves (A'A + Db) x = rhs with preconditioner Minv (csipm_solve's inner solve).
int ew_grid(const void* kernel, long long n) {
    static std::mutex mu;
    static std::vector<std::pair<const void*, int>> cache;   // kernel -> CTAs per wave
    int wave = 0;
    {
        std::lock_guard<std::mutex> lk(mu);
        for (auto& e : cache)
            if (e.first == kernel) { wave = e.second; break; }
        if (!wave) {
            int dev = 0, sms = 0, per_sm = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, EW_THREADS, 0) != cudaSuccess) {
                cudaGetLastError();
                per_sm = 0;
            }
            wave = std::max(1, sms > 0 ? sms : 148) * std::max(1, per_sm);
            cache.emplace_back(kernel, wave);
        }
    }
    const long long b = (n + EW_THREADS - 1) / EW_THREADS;
    return (int)std::max(1LL, std::min(b, (long long)wave));
}

int schur_cg(csipm_handle h, const double* rhs, double* x, bool has_x0, double rtol, int maxit, int* iters,
             const double* r0v, const double* rtol_dev) {
    const long long n = h->N;
    cudaStream_t st = h->stream;
    const double* Minv = h->opt.preconditioner ? h->Minv : nullptr;
    h->resid_kind = RESID_NONE;
    CK(cudaMemsetAsync(h->cgs, 0, sizeof(CgScalars), st));
    const int ppp = passes_per_product(h->g);
    const bool given = has_x0 && r0v != nullptr;
    if (given) {
        rhs = r0v;       // r = rhs - K x0 given: CG on it from x0 with no product
        has_x0 = false;
    } else if (has_x0) {
        EpiCG<double> ep{x, h->Db, h->cg_q, h->ws(h->slots + SL_DUMMY), 0.0};
        CK(solve_AtA(h, x, ep, nullptr, st));
        h->matvecs++;
        h->launches += ppp;
    } else if (!given) {
        CK(cudaMemsetAsync(x, 0, sizeof(double) * n, st));
    }
    ew_launch(cg_init_kernel<double>, n, st, n, rhs, h->cg_q, has_x0 ? 1 : 0, Minv, h->cg_r, h->cg_p,
                                                    h->ws(h->slots + SL_DUMMY), h->cgs, 0.0, DevScalar(rtol, rtol_dev));
    CK(cudaGetLastError());
    h->launches += 1;
    auto iteration = [&](cudaStream_t s, int it) -> cudaError_t {
        EpiCG<double> ep{h->cg_p, h->Db, h->cg_q, h->ws(&h->cgs->pq), 0.0};
        cudaError_t e = solve_AtA(h, h->cg_p, ep, &h->cgs->done, s);
        if (e != cudaSuccess) return e;
        ew_launch(cg_update_kernel<double, double>, n, s, n, it, x, h->cg_r, h->cg_p, h->cg_q, Minv,
                                                                   h->ws(h->slots + SL_DUMMY), h->cgs);
        ew_launch(cg_pupdate_kernel<double>, n, s, n, it, h->cg_r, Minv, h->cg_p, h->cgs);
        return cudaGetLastError();
    };
    // x is a kernel argument: a graph is only valid for the vector it was captured with
    cudaGraphExec_t* ex = x == h->dba ? &h->cg_exec64[0] : (x == h->db ? &h->cg_exec64[1] : nullptr);
    const int r = cg_iterations(h, ex, maxit, iteration, ppp + 2);
    if (r) return r;
    CK(cudaMemcpyAsync(h->hcgs, h->cgs, sizeof(CgScalars), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    h->matvecs += h->hcgs->iters;
    *iters = h->hcgs->iters;
    if (h->hcgs->breakdown) return fail(h, CSIPM_ERR_NONFINITE, "CG breakdown (non-positive curvature or non-finite value)");
    h->resid_kind = RESID_CG64;   // x and r were updated together: r = rhs - K x up to rounding
    if (!h->hcgs->done) return CSIPM_ERR_CG_MAXITER;
    return CSIPM_OK;
}


// ------------------------------------------------------------------ mixed precision
// FP32 PCG corrections on FP64 residuals (iterative refinement of the
// condensed system).  Round 0 solves K d = rhs (or the FP64 residual of the
// warm start x0) in FP32; each later round recomputes r = rhs - K x with the
// FP64 operator and solves K d = r in FP32, asking only for the reduction
// still missing (rtol * |r0| / |r|, floored at MIXED_INNER_RTOL, the level
// FP32 products support).  When the requested rtol is itself at or above the
// floor, round 0 alone answers it (its warm-start residual then comes from
// the FP32 product when rtol >= MIXED_FP32_WARM_RTOL).  An FP32 round stops after
// MIXED_ROUND_MAXIT iterations (stagnation) and the refinement goes on; an
// FP32 breakdown (p.q <= 0 from rounding on a nearly singular direction)
// keeps the partial correction and finishes the solve with FP64 PCG.
constexpr double MIXED_INNER_RTOL = 1e-6;

constexpr double MIXED_FP32_WARM_RTOL = 1e-4;
constexpr int MIXED_ROUND_MAXIT = 100;

// FP64 Db/Minv of the current iterate, when the residual pass left them out
static void ensure_diag64(csipm_handle h) {
    if (!h->diag64_stale) return;
    const long long n = h->N;
    ew_launch(ipm_diag64_kernel, n, h->stream, n, h->s1, h->s2, h->z1, h->z2, h->Db, h->Minv,
                                                                   h->opt.preconditioner);
    h->launches += 1;
    h->diag64_stale = false;
}

int schur_mixed(csipm_handle h, const double* rhs, double* x, bool has_x0, double rtol, int maxit, int* iters,
                const double* r0v, float* xf, bool ready, const double* rin_dev) {
    const long long n = h->N;
    cudaStream_t st = h->stream;
    const bool pc = h->opt.preconditioner != 0;
    const double* Minv = pc ? h->Minv : nullptr;
    const float* Minv32 = pc ? h->f_Minv : nullptr;
    const int ppp = passes_per_product(h->g);
    int total = 0;
    double r0 = -1.0, rn = -1.0;
    // loose Newton tolerances take the warm-start residual from the FP32
    // product: its rounding (~1e-7 relative) is far below what they ask
    // a given warm-start residual serves round 0 with no product at all
    const bool given = has_x0 && (r0v != nullptr || ready);
    const bool fp32_warm = has_x0 && !given && rtol >= MIXED_FP32_WARM_RTOL;
    h->resid_kind = RESID_NONE;
    // with xf, round 0 iterates on xf itself (no correction vector, no FP64
    // accumulation); any FP64 step (refinement, fallback) first takes the
    // iterate into x, and the result goes back to xf at the end
    bool in32 = xf != nullptr;
    auto to64 = [&]() {
        if (!in32) return;
        ew_launch(convert_kernel<float, double>, n, st, n, (const float*)xf, x);
        h->launches += 1;
        in32 = false;
    };
    if (!has_x0) {
        if (in32) CK(cudaMemsetAsync(xf, 0, sizeof(float) * n, st));
        else CK(cudaMemsetAsync(x, 0, sizeof(double) * n, st));
    }
    int status = CSIPM_OK;
    for (int round = 0;; ++round) {
        const double* res = given && round == 0 ? r0v : rhs;
        double rin = std::max(rtol, MIXED_INNER_RTOL);
        if (round > 0 || (has_x0 && !fp32_warm && !given)) {
            to64();
            ensure_diag64(h);
            EpiCG<double> ep{x, h->Db, h->cg_q, h->ws(h->slots + SL_DUMMY), 0.0};
            CK(solve_AtA(h, x, ep, nullptr, st));
            ew_launch(resid64_kernel, n, st, n, rhs, h->cg_q, Minv, h->cg_r, h->ws(h->slots + SL_DOT));
            CK(cudaGetLastError());
            h->matvecs++;
            h->launches += ppp + 1;
            int r = read_slots(h, SL_DOT, 1);
            if (r) return r;
            rn = std::sqrt(h->hslots[SL_DOT]);
            if (!std::isfinite(rn)) return fail(h, CSIPM_ERR_NONFINITE, "non-finite refinement residual");
            if (round == 0) {
                r0 = rn;
            } else {
                if (rn <= rtol * r0 || round > h->opt.ir_max) {
                    h->resid_kind = RESID_CG64;
                    break;
                }
                h->refinements++;
                rin = std::min(0.5, std::max(MIXED_INNER_RTOL, rtol * r0 / rn));
            }
            res = h->cg_r;
        }
        // FP32 PCG on K d = res: from d = 0 into f_x, or (in32) on xf from its start
        float* xi = in32 ? xf : h->f_x;
        const bool started = ready && round == 0 && in32;   // r, p and the CG scalars already written
        if (!started) CK(cudaMemsetAsync(h->cgs, 0, sizeof(CgScalars), st));
        if (!in32) CK(cudaMemsetAsync(h->f_x, 0, sizeof(float) * n, st));
        if (started) {
            // the FP32 CG starts from what the producing kernel wrote
        } else if (round == 0 && fp32_warm) {
            // warm-start residual rhs - K x0 with the FP32 product (x0 rounded to FP32)
            const float* x0f = xf;
            if (!in32) {
                ew_launch(convert_kernel<double, float>, n, st, n, (const double*)x, h->f_p);
                x0f = h->f_p;
            }
            EpiCG<float> ep{x0f, h->f_Db, h->f_q, h->ws(h->slots + SL_DUMMY), 0.0};
            CK(solve_AtA32(h, x0f, ep, nullptr, st));
            h->matvecs++;
            h->launches += ppp + 1;
            ew_launch(cg_init_kernel<float>, n, st, n, rhs, h->f_q, 1, Minv32, h->f_r, h->f_p,
                                                             h->ws(h->slots + SL_DUMMY), h->cgs, 0.0,
                                                             DevScalar(rin, round == 0 ? rin_dev : nullptr));
        } else {
            ew_launch(cg_init_kernel<float>, n, st, n, res, (const float*)nullptr, 0, Minv32, h->f_r, h->f_p,
                                                             h->ws(h->slots + SL_DUMMY), h->cgs, 0.0,
                                                             DevScalar(rin, round == 0 ? rin_dev : nullptr));
        }
        CK(cudaGetLastError());
        if (!started) h->launches += 1;
        const int cap = std::min(maxit, MIXED_ROUND_MAXIT);
        auto iteration = [&](cudaStream_t s, int it) -> cudaError_t {
            EpiCG<float> ep{h->f_p, h->f_Db, h->f_q, h->ws(&h->cgs->pq), 0.0};
            cudaError_t e = solve_AtA32(h, h->f_p, ep, &h->cgs->done, s);
            if (e != cudaSuccess) return e;
            ew_launch(cg_update_kernel<float, float>, n, s, n, it, xi, h->f_r, h->f_p, h->f_q, Minv32,
                                                                    h->ws(h->slots + SL_DUMMY), h->cgs);
            ew_launch(cg_pupdate_kernel<float>, n, s, n, it, h->f_r, Minv32, h->f_p, h->cgs);
            return cudaGetLastError();
        };
        {
            // a graph holds its vectors: one per iterate buffer
            cudaGraphExec_t* ex = xi == h->f_x ? &h->cg_exec32[0]
                                  : (xi == h->f_dba ? &h->cg_exec32[1] : (xi == h->f_db ? &h->cg_exec32[2] : nullptr));
            const int r = cg_iterations(h, ex, cap, iteration, ppp + 2);
            if (r) return r;
        }
        CK(cudaMemcpyAsync(h->hcgs, h->cgs, sizeof(CgScalars), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        h->matvecs += h->hcgs->iters;
        total += h->hcgs->iters;
        if (r0 < 0.0) r0 = rn = std::sqrt(h->hcgs->rz0);   // |rhs| in the M-norm
        if (!in32) {
            ew_launch(add_f32_kernel, n, st, n, h->f_x, x);
            CK(cudaGetLastError());
            h->launches += 1;
        }
        if (h->hcgs->breakdown) {
            to64();
            ensure_diag64(h);
            int its = 0;
            status = schur_cg(h, rhs, x, true, std::min(0.5, rtol * r0 / rn), maxit, &its);
            total += its;
            h->fallbacks++;
            break;
        }
        if (rtol >= MIXED_INNER_RTOL && round == 0 && h->hcgs->done) {
            h->resid_kind = RESID_F32;   // f_r = res - K32 d with x = x0 + d
            break;
        }
    }
    if (xf && !in32) {
        ew_launch(convert_kernel<double, float>, n, st, n, (const double*)x, xf);
        CK(cudaGetLastError());
        h->launches += 1;
    }
    *iters = total;
    return status;
}

// Times each pass of one A^T A product (the CG product: gather -> ... ->
// scatter with the CG epilogue) `reps` times; bytes are the algorithmic
// bytes of the pass (beta-space reals of sizeof(T), spectrum complex of
// 2*sizeof(T), the mask as bits).
template <typename T>
int profile_impl(csipm_handle h, FftOperator<T>& op, const T* x, T* D, T* q, int reps, double* ms_out,
                 double* bytes_out, const char** names, int* npass) {
    const Geom& g = h->g;
    cudaStream_t st = h->stream;
    const double N = (double)g.N, Nh = (double)g.Nh;
    const double w = sizeof(T), cw = 2.0 * sizeof(T), maskb = op.maskw ? N / 8.0 : 0.0;
    const bool f32 = sizeof(T) == 4;
    EpiStore<double> none{nullptr};
    EpiCG<T> ecg{x, D, q, h->ws(h->slots + SL_DUMMY), 0.0};
    const bool mask = op.maskw != nullptr;
    PassArgs<T> ra = op.row_args(1.0 / (2.0 * N), nullptr, nullptr);
    int np = 0;
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
    if (g.dim == 1 && op.l1P) {
        const double M = (double)g.m1;
        r = timeit([&] { return l1d_first(op, x, nullptr, st); }, 2 * w * N + cw * M,
                   f32 ? "fp32 1D lines: gather+C2R+inverse" : "1D lines: gather+C2R+inverse");
        if (r) return r;
        r = timeit([&] { return mask ? l1d_row<T, IN_SPEC, OUT_SPEC, true>(op, ra.scale, nullptr, nullptr, nullptr, st)
                                     : l1d_row<T, IN_SPEC, OUT_SPEC, false>(op, ra.scale, nullptr, nullptr, nullptr, st); },
                   2 * cw * M + maskb, f32 ? "fp32 1D rows: inverse+mask+forward" : "1D rows: inverse+mask+forward");
        if (r) return r;
        r = timeit([&] { return l1d_lines_forward(op, nullptr, st); }, 2 * cw * M,
                   f32 ? "fp32 1D lines: forward" : "1D lines: forward");
        if (r) return r;
        r = timeit([&] { return l1d_post(op, ecg, nullptr, st); }, 2 * cw * M + 3 * w * N,
                   f32 ? "fp32 1D R2C+scatter+CG" : "1D R2C+scatter+CG");
        if (r) return r;
    } else if (g.dim == 1) {
        r = timeit([&] { return mask ? run_row<T, IN_GATHER, OUT_SCATTER, true>(op, ra, x, ecg, st)
                                     : run_row<T, IN_GATHER, OUT_SCATTER, false>(op, ra, x, ecg, st); },
                   4 * w * N + maskb, f32 ? "fp32 row: gather+FFT+scatter+CG" : "row: gather+C2R+mask+R2C+scatter+CG");
        if (r) return r;
    } else {
        // the product's order: beta-side passes along dim 2 (solver-order
        // gather/scatter when the handle uses it), plain ones along dim 3
        PassArgs<T> a2 = op.strided_args(2);
        const bool so = h->sorder;
        if (so && !aligned16(x)) return fail(h, CSIPM_ERR_INVALID, "x must be 16-byte aligned");
        r = timeit([&] { return so ? run_strided<T, true, IN_SGATHER, OUT_SPEC>(op, 2, a2, x, none, st)
                                   : run_strided<T, true, IN_GATHER, OUT_SPEC>(op, 2, a2, x, none, st); },
                   w * N + cw * Nh, f32 ? "fp32 gather+inverse dim2" : "gather+inverse dim2");
        if (r) return r;
        if (g.dim == 3) {
            PassArgs<T> a3 = op.strided_args(3);
            r = timeit([&] { return run_strided<T, true, IN_SPEC, OUT_SPEC>(op, 3, a3, (const double*)nullptr, none, st); },
                       2 * cw * Nh, f32 ? "fp32 inverse dim3" : "inverse dim3");
            if (r) return r;
        }
        r = timeit([&] { return mask ? run_row<T, IN_SPEC, OUT_SPEC, true>(op, ra, (const double*)nullptr, none, st)
                                     : run_row<T, IN_SPEC, OUT_SPEC, false>(op, ra, (const double*)nullptr, none, st); },
                   2 * cw * Nh + maskb, f32 ? "fp32 row: C2R+mask+R2C dim1" : "row: C2R+mask+R2C dim1");
        if (r) return r;
        if (g.dim == 3) {
            PassArgs<T> a3 = op.strided_args(3);
            r = timeit([&] { return run_strided<T, false, IN_SPEC, OUT_SPEC>(op, 3, a3, (const double*)nullptr, none, st); },
                       2 * cw * Nh, f32 ? "fp32 forward dim3" : "forward dim3");
            if (r) return r;
        }
        r = timeit([&] { return so ? run_strided<T, false, IN_SPEC, OUT_SSCATTER>(op, 2, a2, (const double*)nullptr, ecg, st)
                                   : run_strided<T, false, IN_SPEC, OUT_SCATTER>(op, 2, a2, (const double*)nullptr, ecg, st); },
                   cw * Nh + 3 * w * N, f32 ? "fp32 forward dim2+scatter+CG" : "forward dim2+scatter+CG");
        if (r) return r;
    }
    *npass = np;
    return CSIPM_OK;
}


// ------------------------------------------------------------------ IPM state
// The vectors of csipm_solve / csipm_admm (and of csipm_profile_passes),
// allocated on first use from the handle's stream-ordered pool; only the
// missing ones are allocated.
int ensure_ipm_buffers(csipm_handle h) {
    const size_t n_ = (size_t)h->N;
    double** f64[] = {&h->beta, &h->c, &h->s1, &h->s2, &h->z1, &h->z2, &h->rd, &h->Db, &h->Minv, &h->dba, &h->db,
                      &h->cg_r, &h->cg_p, &h->cg_q};
    for (double** q : f64)
        if (!*q && !h->alloc(q, n_)) return fail(h, CSIPM_ERR_OOM, h->err);
    if (h->opt.precision == CSIPM_MIXED) {
        float** f32[] = {&h->f_Db, &h->f_Minv, &h->f_r, &h->f_p, &h->f_q, &h->f_x, &h->f_dba, &h->f_db};
        for (float** q : f32)
            if (!*q && !h->alloc(q, n_)) return fail(h, CSIPM_ERR_OOM, h->err);
    }
    return CSIPM_OK;
}

// ------------------------------------------------------------------ IPM iteration pieces
// What csipm_solve's options make of an iteration.
struct IpmMode {
    bool mixed;
    bool lazy64;      // mixed precision: FP64 barrier diagonals only when a solve asks for them
    bool dir32;       // mixed precision: Newton directions kept in FP32 (f_dba, f_db)
    bool graphable;   // every iteration fits one graph replay (no host decision inside)
};

IpmMode ipm_mode(csipm_handle h) {
    const csipm_options& o = h->opt;
    IpmMode m{};
    m.mixed = o.precision == CSIPM_MIXED;
    // mixed precision with a Newton tolerance the FP32 warm start serves:
    // the FP64 barrier diagonals are only computed when a solve needs them,
    // and the Newton directions stay in FP32 (they are only asked to a
    // relative accuracy >= 1e-4, far above FP32 rounding, and the IPM
    // residual is recomputed in FP64 every iteration)
    m.lazy64 = m.mixed && o.ipm_cg_rtol >= MIXED_FP32_WARM_RTOL;
    m.dir32 = m.lazy64;
    // graph replays: FP64, or mixed with FP32 directions (whose Newton solves
    // are one FP32 CG each: the forcing term's floor is the FP32 round's);
    // refinement rounds and fallbacks decide on the host
    m.graphable = o.cuda_graphs && !o.verbose && (!m.mixed || m.dir32);
    return m;
}

// The residual pass: the pending step on s and z (step), the dual residual,
// the reductions of the stop test, the barrier diagonals and the predictor's
// right-hand side; with FP32 directions also the start of the predictor's
// FP32 CG at the tolerance *crtol.
cudaError_t launch_resid_pass(csipm_handle h, cudaStream_t st, const IpmMode& md, bool step, const double* crtol) {
    const long long n = h->N;
    const double lam = h->lambda;
    const bool pc = h->opt.preconditioner != 0;
    const double* bv = h->sorder ? h->bs : h->b;
    if (md.dir32)
        ew_launch(ipm_resdiag_kernel<float, float>, n, st, n, bv, h->Qb, lam, h->beta, h->s1, h->s2, h->z1, h->z2,
                  step ? h->f_dba : nullptr, step ? h->f_db : nullptr, h->slots + SL_SIGMU, h->slots + SL_ALPHA,
                  h->rd, (double*)nullptr, (double*)nullptr, h->f_Db, h->f_Minv, pc ? 1 : 0, h->rhs,
                  h->ws(h->slots + SL_RED), h->f_r, h->f_p, h->cgs, DevScalar(0.0, crtol));
    else
        ew_launch(ipm_resdiag_kernel<float, double>, n, st, n, bv, h->Qb, lam, h->beta, h->s1, h->s2, h->z1, h->z2,
                  step ? h->dba : nullptr, step ? h->db : nullptr, h->slots + SL_SIGMU, h->slots + SL_ALPHA,
                  h->rd, md.lazy64 ? nullptr : h->Db, md.lazy64 ? nullptr : h->Minv,
                  md.mixed ? h->f_Db : nullptr, md.mixed ? h->f_Minv : nullptr, pc ? 1 : 0, h->rhs,
                  h->ws(h->slots + SL_RED), (float*)nullptr, (float*)nullptr, (CgScalars*)nullptr, DevScalar());
    return cudaGetLastError();
}

// The corrector's right-hand side after the predictor's step statistics and
// centring target; rk says where the predictor left its residual (RESID_*),
// from which the corrector's warm-start residual is formed with no product.
// FP32 directions with a known residual: this pass also starts the
// corrector's FP32 CG (r, p, scalars) at the tolerance *crtol.
cudaError_t launch_corrector_rhs(csipm_handle h, cudaStream_t st, const IpmMode& md, int rk, const double* crtol) {
    const long long n = h->N;
    const double lam = h->lambda;
    const float* rp32 = rk == RESID_F32 ? h->f_r : nullptr;
    const double* rp64 = rk == RESID_CG64 ? h->cg_r : nullptr;
    const double* sigmu_d = h->slots + SL_SIGMU;
    const bool cstart = md.dir32 && rk != RESID_NONE;
    float* cr = cstart ? h->f_r : nullptr;
    float* cp = cstart ? h->f_p : nullptr;
    const float* cm = h->opt.preconditioner ? h->f_Minv : nullptr;
    RedWorkspace cws = h->ws(h->slots + SL_DUMMY);
    if (md.dir32 && rp32)
        ew_launch(ipm_rhs_kernel<float, float>, n, st, n, lam, h->s1, h->s2, h->z1, h->z2, h->rd,
                  (const float*)h->f_dba, sigmu_d, h->rhs, rp32, h->f_db, cr, cp, cm, h->cgs, cws,
                  DevScalar(0.0, crtol));
    else if (md.dir32)
        ew_launch(ipm_rhs_kernel<double, float>, n, st, n, lam, h->s1, h->s2, h->z1, h->z2, h->rd,
                  (const float*)h->f_dba, sigmu_d, h->rhs, rp64, h->f_db, cr, cp, cm, h->cgs, cws,
                  DevScalar(0.0, crtol));
    else if (rp32)
        ew_launch(ipm_rhs_kernel<float, double>, n, st, n, lam, h->s1, h->s2, h->z1, h->z2, h->rd,
                  (const double*)h->dba, sigmu_d, h->rhs, rp32, h->db, (float*)nullptr, (float*)nullptr,
                  (const float*)nullptr, (CgScalars*)nullptr, cws, DevScalar());
    else
        ew_launch(ipm_rhs_kernel<double, double>, n, st, n, lam, h->s1, h->s2, h->z1, h->z2, h->rd,
                  (const double*)h->dba, sigmu_d, h->rhs, rp64, h->db, (float*)nullptr, (float*)nullptr,
                  (const float*)nullptr, (CgScalars*)nullptr, cws, DevScalar());
    return cudaGetLastError();
}

// After the corrector: its step statistics, the step length and the beta
// step (s and z take the same step inside the next residual pass).
cudaError_t launch_step(csipm_handle h, cudaStream_t st, const IpmMode& md) {
    const long long n = h->N;
    const double lam = h->lambda;
    const double* sigmu_d = h->slots + SL_SIGMU;
    double* alpha_d = h->slots + SL_ALPHA;
    if (md.dir32)
        ew_launch(ipm_stepstats_kernel<float>, n, st, n, lam, h->s1, h->s2, h->z1, h->z2, (const float*)h->f_dba,
                  sigmu_d, (const float*)h->f_db, h->ws(h->slots + SL_SS));
    else
        ew_launch(ipm_stepstats_kernel<double>, n, st, n, lam, h->s1, h->s2, h->z1, h->z2, (const double*)h->dba,
                  sigmu_d, (const double*)h->db, h->ws(h->slots + SL_SS));
    ipm_alpha_kernel<<<1, 1, 0, st>>>(h->slots + SL_SS, h->ctl, alpha_d);
    if (md.dir32)
        ew_launch(ipm_beta_step_kernel<float>, n, st, n, h->beta, (const float*)h->f_db, (const double*)alpha_d);
    else
        ew_launch(ipm_beta_step_kernel<double>, n, st, n, h->beta, (const double*)h->db, (const double*)alpha_d);
    return cudaGetLastError();
}

// ------------------------------------------------------------------ IPM iteration graph
// Adds a conditional node to the graph stream s is capturing: a handle on
// that graph, set_fn(s, hnd) captured before the node (the kernel that sets
// the handle each time the node is reached), the node itself, then
// body_fn(s2, hnd) captured into the node's body on stream s2.  Afterwards s
// depends on the node.
template <class SetFn, class BodyFn>
bool capture_conditional(cudaStream_t s, cudaStream_t s2, cudaGraphConditionalNodeType type, SetFn&& set_fn,
                         BodyFn&& body_fn) {
    cudaStreamCaptureStatus cst;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    if (cudaStreamGetCaptureInfo(s, &cst, nullptr, &g, &deps, &nd) != cudaSuccess || cst != cudaStreamCaptureStatusActive)
        return false;
    cudaGraphConditionalHandle hnd = 0;
    if (cudaGraphConditionalHandleCreate(&hnd, g, 0, 0) != cudaSuccess) return false;
    if (!set_fn(s, hnd)) return false;
    if (cudaStreamGetCaptureInfo(s, &cst, nullptr, &g, &deps, &nd) != cudaSuccess) return false;
    cudaGraphNodeParams p = {};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = hnd;
    p.conditional.type = type;
    p.conditional.size = 1;
    cudaGraphNode_t node = nullptr;
    if (cudaGraphAddNode(&node, g, deps, nd, &p) != cudaSuccess) return false;
    cudaGraph_t body = p.conditional.phGraph_out[0];
    if (cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies) != cudaSuccess) return false;
    if (cudaStreamBeginCaptureToGraph(s2, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return false;
    const bool ok = body_fn(s2, hnd);
    cudaGraph_t out = nullptr;
    const bool ended = cudaStreamEndCapture(s2, &out) == cudaSuccess;
    return ok && ended;
}

// The graph of whole interior-point iterations (FP64, or mixed precision
// with FP32 directions): a conditional WHILE node whose body is the rest of
// one iteration after its stop test — predictor CG (a nested WHILE node),
// then, if it converged, the step statistics, centring target, corrector
// right-hand side and corrector CG, then, if that converged, the step, the
// next A'A product, the next residual pass and its stop test, which keeps
// the outer loop going while the method runs.  A CG breakdown, or a loop cap
// below the solve's, ends the replay with the iteration handed back to the
// host (IPM_ABORT).  Captured once per handle.
bool build_ipm_graph(csipm_handle h, const IpmMode& md) {
    const long long n = h->N;
    const int maxit = h->opt.cg_maxit;
    const bool pc = h->opt.preconditioner != 0;
    const double* Minv = pc ? h->Minv : nullptr;
    const float* Minv32 = pc ? h->f_Minv : nullptr;
    // an FP32 round that is not done at its cap goes on to FP64 refinement on
    // the host; an FP64 loop that reached the solve's own cap is accepted, as
    // the plain loop accepts it
    const int cap = md.dir32 ? std::min(maxit, MIXED_ROUND_MAXIT) : std::min(maxit, CG_WHILE_CAP);
    const int cap_is_limit = (!md.dir32 && cap >= maxit) ? 1 : 0;
    const double* rt_dev = &h->ctl->rt;
    int kernels = 0;
    cudaStream_t ss[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    for (auto& x : ss)
        if (cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking) != cudaSuccess) x = nullptr;
    cudaGraph_t graph = nullptr;
    bool ok = ss[4] != nullptr && cudaGraphCreate(&graph, 0) == cudaSuccess;
    cudaGraphConditionalHandle loop = 0;
    cudaGraphNodeParams lp = {};
    cudaGraphNode_t lnode = nullptr;
    if (ok) ok = cudaGraphConditionalHandleCreate(&loop, graph, 1, cudaGraphCondAssignDefault) == cudaSuccess;
    if (ok) {
        lp.type = cudaGraphNodeTypeConditional;
        lp.conditional.handle = loop;
        lp.conditional.type = cudaGraphCondTypeWhile;
        lp.conditional.size = 1;
        ok = cudaGraphAddNode(&lnode, graph, nullptr, 0, &lp) == cudaSuccess;
    }
    // one CG loop over the iterate x (FP64) or xf (FP32)
    auto cg_loop = [&](cudaStream_t s, cudaStream_t sb, double* x, float* xf) -> bool {
        auto arm = [&](cudaStream_t q, cudaGraphConditionalHandle hc) {
            cg_arm_kernel<<<1, 1, 0, q>>>(hc, h->cgs);
            ++kernels;
            return cudaGetLastError() == cudaSuccess;
        };
        auto body = [&](cudaStream_t q, cudaGraphConditionalHandle hc) {
            for (int it = 0; it < 2; ++it) {
                cudaError_t e;
                if (md.dir32) {
                    EpiCG<float> ep{h->f_p, h->f_Db, h->f_q, h->ws(&h->cgs->pq), 0.0};
                    e = solve_AtA32(h, h->f_p, ep, &h->cgs->done, q);
                    if (e != cudaSuccess) return false;
                    ew_launch(cg_update_kernel<float, float>, n, q, n, it, xf, h->f_r, h->f_p, h->f_q, Minv32,
                              h->ws(h->slots + SL_DUMMY), h->cgs);
                    ew_launch(cg_pupdate_kernel<float>, n, q, n, it, h->f_r, Minv32, h->f_p, h->cgs);
                } else {
                    EpiCG<double> ep{h->cg_p, h->Db, h->cg_q, h->ws(&h->cgs->pq), 0.0};
                    e = solve_AtA(h, h->cg_p, ep, &h->cgs->done, q);
                    if (e != cudaSuccess) return false;
                    ew_launch(cg_update_kernel<double, double>, n, q, n, it, x, h->cg_r, h->cg_p, h->cg_q, Minv,
                              h->ws(h->slots + SL_DUMMY), h->cgs);
                    ew_launch(cg_pupdate_kernel<double>, n, q, n, it, h->cg_r, Minv, h->cg_p, h->cgs);
                }
            }
            cg_continue_kernel<<<1, 1, 0, q>>>(hc, h->cgs, cap);
            return cudaGetLastError() == cudaSuccess;
        };
        return capture_conditional(s, sb, cudaGraphCondTypeWhile, arm, body);
    };
    auto check = [&](int which, cudaGraphConditionalHandle hi, cudaStream_t q) {
        ipm_cg_check_kernel<<<1, 1, 0, q>>>(h->cgs, h->ctl, which, cap_is_limit, hi, loop);
        ++kernels;
        return cudaGetLastError() == cudaSuccess;
    };
    if (ok) ok = cudaStreamBeginCaptureToGraph(ss[0], lp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                               cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    if (ok) {
        cudaStream_t s0 = ss[0];
        // ---- predictor from zero: FP32 directions start from the residual
        // pass's CG start, FP64 ones from r = rhs
        if (!md.dir32) {
            ew_launch(fill_kernel, n, s0, n, 0.0, h->dba);
            ew_launch(cg_init_kernel<double>, n, s0, n, (const double*)h->rhs, (const double*)nullptr, 0, Minv,
                      h->cg_r, h->cg_p, h->ws(h->slots + SL_DUMMY), h->cgs, 0.0, DevScalar(0.0, rt_dev));
            kernels += 2;
        } else {
            ew_launch(fill_f32_kernel, n, s0, n, 0.0f, h->f_dba);
            kernels += 1;
        }
        ok = cg_loop(s0, ss[4], h->dba, h->f_dba);
        ok = ok && capture_conditional(
                       s0, ss[1], cudaGraphCondTypeIf, [&](cudaStream_t q, cudaGraphConditionalHandle hi) { return check(1, hi, q); },
                       [&](cudaStream_t s1, cudaGraphConditionalHandle) -> bool {
                           // ---- corrector
                           if (md.dir32)
                               ew_launch(ipm_stepstats_kernel<float>, n, s1, n, h->lambda, h->s1, h->s2, h->z1, h->z2,
                                         (const float*)nullptr, (const double*)nullptr, h->f_dba,
                                         h->ws(h->slots + SL_SS));
                           else
                               ew_launch(ipm_stepstats_kernel<double>, n, s1, n, h->lambda, h->s1, h->s2, h->z1,
                                         h->z2, (const double*)nullptr, (const double*)nullptr, h->dba,
                                         h->ws(h->slots + SL_SS));
                           ipm_sigma_kernel<<<1, 1, 0, s1>>>(h->slots + SL_SS, h->ctl, h->slots + SL_SIGMU);
                           if (launch_corrector_rhs(h, s1, md, md.dir32 ? RESID_F32 : RESID_CG64, &h->ctl->rin) !=
                               cudaSuccess)
                               return false;
                           kernels += 3;
                           if (!md.dir32) {
                               // r = rhs_c - K dba (written to rd by the rhs pass), from x = dba
                               ew_launch(cg_init_kernel<double>, n, s1, n, (const double*)h->rd, (const double*)nullptr,
                                         0, Minv, h->cg_r, h->cg_p, h->ws(h->slots + SL_DUMMY), h->cgs, 0.0,
                                         DevScalar(0.0, rt_dev));
                               ++kernels;
                           }
                           if (!cg_loop(s1, ss[4], h->db, h->f_db)) return false;
                           return capture_conditional(
                               s1, ss[2], cudaGraphCondTypeIf,
                               [&](cudaStream_t q, cudaGraphConditionalHandle hi) { return check(2, hi, q); },
                               [&](cudaStream_t s2, cudaGraphConditionalHandle) -> bool {
                                   // ---- step, next product, next residual pass and stop test
                                   if (launch_step(h, s2, md) != cudaSuccess) return false;
                                   EpiStore<double> ep{h->Qb};
                                   if (solve_AtA(h, h->beta, ep, nullptr, s2) != cudaSuccess) return false;
                                   if (launch_resid_pass(h, s2, md, true, &h->ctl->rin_next) != cudaSuccess)
                                       return false;
                                   ipm_stop_kernel<<<1, 1, 0, s2>>>(h->slots + SL_RED, h->ctl, 1, loop);
                                   kernels += 3 + passes_per_product(h->g) + 2;
                                   return cudaGetLastError() == cudaSuccess;
                               });
                       });
        cudaGraph_t out = nullptr;
        ok = cudaStreamEndCapture(ss[0], &out) == cudaSuccess && ok;
    }
    if (ok) ok = cudaGraphInstantiate(&h->ipm_exec, graph, 0) == cudaSuccess;
    for (auto& x : ss)
        if (x) cudaStreamDestroy(x);
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    if (!ok) h->ipm_exec = nullptr;
    h->ipm_body_kernels = kernels;
    return ok;
}

// Runs the iteration graph from the current iterate (its residual pass and
// stop test done, the method still running).  Returns 0 with the control
// block read back (status: stopped, or IPM_ABORT with the iteration handed
// back), 1 when no graph could be built, or a (negative) csipm_status.
int ipm_graph_run(csipm_handle h, const IpmMode& md, csipm_stats* S) {
    if (!h->ipm_exec && !build_ipm_graph(h, md)) {
        h->ipm_graph_off = true;
        return 1;
    }
    cudaStream_t st = h->stream;
    h->hctl->cg_iter = 0;
    h->hctl->graph_iters = 0;
    CK(cudaMemcpyAsync(&h->ctl->cg_iter, &h->hctl->cg_iter, 2 * sizeof(int), cudaMemcpyHostToDevice, st));
    CK(cudaGraphLaunch(h->ipm_exec, st));
    CK(cudaMemcpyAsync(h->hctl, h->ctl, sizeof(IpmCtl), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    const IpmCtl& C = *h->hctl;
    S->cg_iter += C.cg_iter;
    S->graph_iters += C.graph_iters;
    // one product per CG iteration plus the residual product of every completed body
    h->matvecs += C.cg_iter + C.graph_iters;
    const int ppp = passes_per_product(h->g);
    h->launches += 1 + (long long)C.graph_iters * h->ipm_body_kernels + (long long)C.cg_iter * (ppp + 2) +
                   (C.cg_iter + 1) / 2;
    return CSIPM_OK;
}

}  // namespace csipm_internal

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
    opt->cuda_graphs = 1;
    opt->autotune = 1;
    opt->stream = nullptr;
    opt->ipm_cg_forcing = 100.0;
    return CSIPM_OK;
}

const char* csipm_last_error(csipm_handle h) {
    return h ? h->err.c_str() : get_last_error();
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
    if (h->opt.precision != CSIPM_FP64 && h->opt.precision != CSIPM_MIXED) {
        delete h;
        return fail(nullptr, CSIPM_ERR_INVALID, "precision must be CSIPM_FP64 or CSIPM_MIXED");
    }
    cudaGetDevice(&h->device);
    int n[3] = {prob->size[0], prob->dim >= 2 ? prob->size[1] : 1, prob->dim >= 3 ? prob->size[2] : 1};
    h->g = make_geom(prob->dim, n, n[0] / 2 + 1);
    h->N = h->g.N;
    h->lambda = prob->lambda;
    h->z0 = prob->z0;
    if (h->opt.cg_maxit <= 0) h->opt.cg_maxit = (int)std::min<long long>(2 * h->N, 1 << 30);
    auto bail = [&](int st, const std::string& m) { g_last_error = m; delete h; return st; };
    // NULL selects the CUDA default stream (the cuBLAS/cuFFT convention)
    h->stream = (cudaStream_t)h->opt.stream;
    h->own_stream = false;
    h->pool = device_pool(h->device);
    if (!h->pool) return bail(CSIPM_ERR_CUDA, "device memory pool creation failed");
    h->op64.pool = h->pool;
    h->op32.pool = h->pool;
    // mask: indices checked here, bits built on the device from a stream-ordered copy
    int64_t* dmiss = nullptr;
    const int64_t nm = prob->n_missing > 0 ? prob->n_missing : 0;
    if (nm > 0) {
        if (!prob->host_missing) return bail(CSIPM_ERR_INVALID, "host_missing is null");
        for (int64_t t = 0; t < nm; ++t) {
            const int64_t idx = prob->host_missing[t];
            if (idx < 0 || idx >= h->N) return bail(CSIPM_ERR_INVALID, "missing index out of range");
        }
        if (cudaMallocFromPoolAsync((void**)&dmiss, sizeof(int64_t) * nm, h->pool, h->stream) != cudaSuccess)
            return bail(CSIPM_ERR_OOM, "out of device memory (missing indices)");
        // through a pinned bounce buffer the handle keeps (an asynchronous
        // copy: a pageable one would pass through the driver's shared staging);
        // pageable when no pinned memory is left
        const void* src = prob->host_missing;
        size_t pb = 1 << 16;
        while (pb < sizeof(int64_t) * (size_t)nm) pb <<= 1;
        if ((h->hmiss = pinned_get(pb)) != nullptr) {
            h->hmiss_bytes = pb;
            std::memcpy(h->hmiss, prob->host_missing, sizeof(int64_t) * (size_t)nm);
            src = h->hmiss;
        }
        if (cudaMemcpyAsync(dmiss, src, sizeof(int64_t) * nm, cudaMemcpyHostToDevice, h->stream) != cudaSuccess) {
            cudaFreeAsync(dmiss, h->stream);
            return bail(CSIPM_ERR_CUDA, "missing-index upload failed");
        }
    }
    const bool mixed = h->opt.precision == CSIPM_MIXED;
    bool ok = h->op64.init(h->g, dmiss, nm, h->stream, &err);
    if (ok) h->bytes += h->op64.bytes;
    if (ok && mixed) {
        ok = h->op32.init(h->g, dmiss, nm, h->stream, &err);
        if (ok) h->bytes += h->op32.bytes;
    }
    if (dmiss) cudaFreeAsync(dmiss, h->stream);
    if (!ok) return bail(err.find("memory") != std::string::npos ? CSIPM_ERR_OOM : CSIPM_ERR_UNSUPPORTED, err);
    if (h->opt.autotune) {
        autotune(h->op64, h->stream);
        if (mixed) autotune(h->op32, h->stream);
    }
    // reduction workspace: enough partials for the largest grid
    size_t maxblocks = 8192;
    if (h->g.dim >= 2)
        maxblocks = std::max<size_t>(maxblocks, (size_t)((h->g.m1 + FFT2_TB_MIN) / FFT2_TB_MIN) * (h->g.dim == 3 ? h->g.n3 : 1));
    if (h->g.dim >= 3) maxblocks = std::max<size_t>(maxblocks, (size_t)((h->g.m1 + FFT2_TB_MIN) / FFT2_TB_MIN) * h->g.n2);
    maxblocks = std::max<size_t>(maxblocks, (size_t)h->op64.row_cfg.grid.x);
    if (h->g.dim >= 2) maxblocks = std::max<size_t>(maxblocks, (size_t)h->op64.s2_cfg.grid.x * h->op64.s2_cfg.grid.y);
    if (h->g.dim >= 3) maxblocks = std::max<size_t>(maxblocks, (size_t)h->op64.s3_cfg.grid.x * h->op64.s3_cfg.grid.y);
    const size_t n_ = (size_t)h->N;
    // the interior-point state is allocated by the first csipm_solve /
    // csipm_admm (ensure_ipm_buffers): a handle used as an operator or a KKT
    // plugin holds only the operator, A^T z0 and two scratch vectors
    if (!h->alloc(&h->partials, maxblocks * 8) || !h->alloc(&h->ticket, 1) || !h->alloc(&h->slots, SL_COUNT) ||
        !h->alloc(&h->cgs, 1) || !h->alloc(&h->ctl, 1) || !h->alloc(&h->b, n_) || !h->alloc(&h->Qb, n_) ||
        !h->alloc(&h->rhs, n_))
        return bail(CSIPM_ERR_OOM, h->err);
    static_assert(sizeof(double) * SL_COUNT == csipm_handle_s::HSLOT_BYTES, "slot block size");
    static_assert(sizeof(CgScalars) <= csipm_handle_s::HCGS_BYTES, "CG scalar block size");
    static_assert(sizeof(IpmCtl) <= csipm_handle_s::HCTL_BYTES, "IPM control block size");
    h->hslots = (double*)pinned_get(csipm_handle_s::HSLOT_BYTES);
    h->hcgs = (CgScalars*)pinned_get(csipm_handle_s::HCGS_BYTES);
    h->hctl = (IpmCtl*)pinned_get(csipm_handle_s::HCTL_BYTES);
    if (!h->hslots || !h->hcgs || !h->hctl) return bail(CSIPM_ERR_OOM, "pinned host allocation failed");
    cudaMemsetAsync(h->ticket, 0, sizeof(unsigned int), h->stream);
    cudaMemsetAsync(h->slots, 0, sizeof(double) * SL_COUNT, h->stream);
    cudaEventCreate(&h->ev0);
    cudaEventCreate(&h->ev1);
    cudaEventCreate(&h->ev_rp[0]);
    cudaEventCreate(&h->ev_rp[1]);
    // A^T z0 (src/fft_model.jl:60-62) and ||z0||^2
    EpiStore<double> st_b{h->b};
    {
        cudaError_t e0 = op_At(h->op64, prob->z0, st_b, h->stream);
        if (e0 != cudaSuccess) return bail(CSIPM_ERR_CUDA, std::string("A^T z0 failed: ") + cudaGetErrorString(e0));
    }
    // ||z0||^2 stays on the device (csipm_solve's stop test reads it there)
    ew_launch(dot2_kernel, h->N, h->stream, h->N, prob->z0, prob->z0, nullptr, nullptr, h->ws(h->slots + SL_Z0SQ));
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return bail(CSIPM_ERR_CUDA, std::string("CUDA: ") + cudaGetErrorString(e));
    if (h->opt.layout == 0 && solver_order_ok(h->op64) && (!mixed || solver_order_ok(h->op32))) {
        if (!h->alloc(&h->bs, n_)) return bail(CSIPM_ERR_OOM, h->err);
        // plane map: the entries of the planes i = 0 and i = M1 in solver
        // order, built on the device (no host loop, no copy)
        const Geom& g = h->g;
        const size_t np = (size_t)2 * g.n2 * g.n3;
        if (!h->alloc(&h->pmap, np)) return bail(CSIPM_ERR_OOM, h->err);
        plane_map_kernel<<<ew_blocks((long long)np), EW_THREADS, 0, h->stream>>>(g, h->pmap);
        h->op64.pmap = h->pmap;
        h->op32.pmap = h->pmap;
        if (cudaGetLastError() != cudaSuccess || to_solver_order(h->g, h->b, h->bs, h->stream) != cudaSuccess)
            return bail(CSIPM_ERR_CUDA, "solver-order set-up failed");
        h->sorder = true;
    }
    *out = h;
    return CSIPM_OK;
}

int csipm_trim_pool(int device) {
    int dev = device;
    if (dev < 0 && cudaGetDevice(&dev) != cudaSuccess) return CSIPM_ERR_NO_DEVICE;
    cudaMemPool_t pool = device_pool(dev);
    if (!pool) return fail(nullptr, CSIPM_ERR_CUDA, "device memory pool unavailable");
    if (cudaMemPoolTrimTo(pool, 0) != cudaSuccess) return fail(nullptr, CSIPM_ERR_CUDA, "cudaMemPoolTrimTo failed");
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

int csipm_solve(csipm_handle h, double* beta_out, double* c_out, csipm_stats* stats) {
    if (!h || !beta_out) return fail(h, CSIPM_ERR_INVALID, "null argument");
    {
        const int r = ensure_ipm_buffers(h);
        if (r) return r;
    }
    const long long n = h->N;
    cudaStream_t st = h->stream;
    const double lam = h->lambda;
    const csipm_options& o = h->opt;
    csipm_stats S{};
    const int mv0 = h->matvecs;
    const int rf0 = h->refinements;
    const int fb0 = h->fallbacks;
    const long long la0 = h->launches;
    const bool mixed = o.precision == CSIPM_MIXED;
    const int ppp = passes_per_product(h->g);
    const IpmMode md = ipm_mode(h);
    const bool lazy64 = md.lazy64, dir32 = md.dir32;
    cudaEventRecord(h->ev0, st);
    const double* bv = h->sorder ? h->bs : h->b;
    // ---- initial point: beta = soft(A^T z0, lambda), z from the clipped gradient, c balanced
    ew_launch(ipm_init1_kernel, n, st, n, bv, lam, h->beta, h->ws(h->slots + SL_MAXB));
    CK(cudaGetLastError());
    {
        EpiStore<double> ep{h->Qb};
        CK(solve_AtA(h, h->beta, ep, nullptr, st));
        h->matvecs++;
    }
    h->launches += 2 + ppp;
    ew_launch(ipm_init2_kernel, n, st, n, bv, h->Qb, lam, h->beta, h->slots + SL_MAXB, h->s1, h->s2, h->z1,
                                                 h->z2);
    CK(cudaGetLastError());
    {
        int r0 = read_slots(h, SL_MAXB, 2);
        if (r0) return r0;
    }
    // ---- the device control block: stop test and Newton tolerances
    {
        IpmCtl& c = *h->hctl;
        std::memset(&c, 0, sizeof(IpmCtl));
        c.tol = o.tol;
        c.rt_opt = o.ipm_cg_rtol;
        c.forcing = o.ipm_cg_forcing;
        c.rt_floor = CG_FORCING_FLOOR;
        c.rin_floor = MIXED_INNER_RTOL;
        c.z0sq = 0.0;   // copied from the device slot below
        c.kkt_scale = std::max(1.0, h->hslots[SL_MAXB + 1]);
        c.lam = lam;
        c.two_n = 2.0 * (double)n;
        c.max_iter = o.max_iter;
        c.k = -1;
        c.rt_next = o.ipm_cg_rtol;   // iteration 0 solves at the option
        c.rin_next = std::max(o.ipm_cg_rtol, MIXED_INNER_RTOL);
        c.status = IPM_RUNNING;
        CK(cudaMemcpyAsync(h->ctl, h->hctl, sizeof(IpmCtl), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(&h->ctl->z0sq, h->slots + SL_Z0SQ, sizeof(double), cudaMemcpyDeviceToDevice, st));
    }
    const double* rt_dev = &h->ctl->rt;
    const double* rin_dev = &h->ctl->rin;
    int status = CSIPM_ERR_IPM_MAXITER;
    bool pending = false;    // a beta step whose slack / multiplier step waits for the next residual pass
    bool qb_valid = true;    // Qb = A'A beta of the current beta (the initial point's product)
    bool resume = false;     // a graph replay handed an iteration back: rerun its residual pass only
    bool use_graph = md.graphable && !h->ipm_graph_off;
    for (;;) {
        if (!qb_valid) {
            EpiStore<double> ep{h->Qb};
            CK(solve_AtA(h, h->beta, ep, nullptr, st));
            h->matvecs++;
            h->launches += ppp;
        }
        qb_valid = false;
        h->diag64_stale = lazy64;
        {
            // algorithmic bytes: b, Qb, beta, s1, s2, z1, z2 read; rd, rhs written;
            // with the pending step the two directions read and s, z written;
            // the barrier diagonals written in FP64 and/or FP32; with FP32
            // directions the predictor CG's r and p written
            const double td = dir32 ? 4.0 : 8.0;
            const double per = 56.0 + 16.0 + (pending ? 2.0 * td + 32.0 : 0.0) + (lazy64 ? 0.0 : 16.0) +
                               (mixed ? 8.0 : 0.0) + (dir32 ? 8.0 : 0.0);
            S.resid_pass_bytes += per * (double)n;
            S.resid_pass_launches += 1;
        }
        cudaEventRecord(h->ev_rp[0], st);
        // a resumed iteration restarts its predictor at this iteration's tolerance
        CK(launch_resid_pass(h, st, md, pending, resume ? rin_dev : &h->ctl->rin_next));
        cudaEventRecord(h->ev_rp[1], st);
        pending = false;
        h->launches += 1;
        if (!resume) {
            ipm_stop_kernel<<<1, 1, 0, st>>>(h->slots + SL_RED, h->ctl, 0, 0);
            CK(cudaGetLastError());
            h->launches += 1;
        }
        resume = false;
        CK(cudaMemcpyAsync(h->hctl, h->ctl, sizeof(IpmCtl), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        {
            float rp_ms = 0.f;   // the stream is synchronised: both events are complete
            if (cudaEventElapsedTime(&rp_ms, h->ev_rp[0], h->ev_rp[1]) == cudaSuccess) S.resid_pass_ms += rp_ms;
        }
        const IpmCtl& C = *h->hctl;
        if (o.verbose)
            std::fprintf(stderr, "csipm it %3d  mu %.3e  gap %.3e  |rd| %.2e  obj %.12e  rtol %.1e  cg %d\n", C.k, C.mu,
                         C.gap, C.dual_inf, C.F, C.rt, S.cg_iter);
        if (C.status != IPM_RUNNING) break;
        if (use_graph) {
            // every further iteration inside one graph launch: no host round trip
            // until the method stops or a Newton solve needs the host
            const int g = ipm_graph_run(h, md, &S);
            if (g == 1) {   // the graph could not be built: plain launches from here on
                use_graph = false;
            } else if (g) {
                return g;
            } else if (h->hctl->status == IPM_ABORT) {
                use_graph = false;
                resume = true;       // Qb is current and no step is pending
                qb_valid = true;
                h->hctl->status = IPM_RUNNING;
                CK(cudaMemcpyAsync(&h->ctl->status, &h->hctl->status, sizeof(int), cudaMemcpyHostToDevice, st));
                continue;
            } else {
                break;
            }
        }
        const double rt = C.rt;                               // this iteration's Newton tolerance (host copy)
        const double cg_rin = C.rin;
        // ---- predictor (affine scaling): diagonals and right-hand side came with the residual
        int its = 0;
        int cs = mixed ? schur_mixed(h, h->rhs, h->dba, false, rt, o.cg_maxit, &its, nullptr,
                                     dir32 ? h->f_dba : nullptr, dir32, rin_dev)
                       : schur_cg(h, h->rhs, h->dba, false, rt, o.cg_maxit, &its, nullptr, rt_dev);
        S.cg_iter += its;
        if (cs != CSIPM_OK && cs != CSIPM_ERR_CG_MAXITER) { status = cs; break; }
        // the centring target and the step length are computed on the device
        // from the step statistics: no host round trip inside the iteration
        if (dir32)
            ew_launch(ipm_stepstats_kernel<float>, n, st, n, lam, h->s1, h->s2, h->z1, h->z2, (const float*)nullptr,
                      (const double*)nullptr, h->f_dba, h->ws(h->slots + SL_SS));
        else
            ew_launch(ipm_stepstats_kernel<double>, n, st, n, lam, h->s1, h->s2, h->z1, h->z2,
                      (const double*)nullptr, (const double*)nullptr, h->dba, h->ws(h->slots + SL_SS));
        ipm_sigma_kernel<<<1, 1, 0, st>>>(h->slots + SL_SS, h->ctl, h->slots + SL_SIGMU);
        // ---- corrector, warm-started at dba.  Its starting residual
        // rhs_c - K dba = rhs_c - rhs_p + (rhs_p - K dba) comes from the
        // predictor solve's residual (kept by CG's recurrence) with no
        // product; mixed precision at tight Newton tolerances computes it
        // with an FP64 product instead, as refinement wants.
        const int rk = (!mixed || o.ipm_cg_rtol >= MIXED_FP32_WARM_RTOL) ? h->resid_kind : RESID_NONE;
        CK(launch_corrector_rhs(h, st, md, rk, rin_dev));
        const bool cstart = dir32 && rk != RESID_NONE;
        const double* r0v = rk != RESID_NONE && !cstart ? h->rd : nullptr;
        cs = mixed ? schur_mixed(h, h->rhs, h->db, true, rt, o.cg_maxit, &its, r0v, dir32 ? h->f_db : nullptr,
                                 cstart, rin_dev)
                   : schur_cg(h, h->rhs, h->db, true, rt, o.cg_maxit, &its, r0v, rt_dev);
        S.cg_iter += its;
        if (cs != CSIPM_OK && cs != CSIPM_ERR_CG_MAXITER) { status = cs; break; }
        (void)cg_rin;
        CK(launch_step(h, st, md));
        h->launches += 6;   // sigma, corrector rhs, 2 step statistics, alpha, beta step (+ the Newton solves' launches)
        pending = true;
    }
    {
        const IpmCtl& C = *h->hctl;
        if (status == CSIPM_ERR_IPM_MAXITER) {   // no solver error: the control block says why the loop ended
            if (C.status == IPM_CONVERGED) status = CSIPM_OK;
            else if (C.status == IPM_NONFINITE) status = fail(h, CSIPM_ERR_NONFINITE, "non-finite iterate");
        }
        S.obj = C.obj;
        S.lasso_obj = C.F;
        S.dual_inf = C.dual_inf;
        S.mu = C.mu;
        S.gap = C.gap;
        S.ipm_iter = C.k;
    }
    if (c_out) {
        ew_launch(half_sum_kernel, n, st, n, h->s1, h->s2, h->c);
        CK(cudaGetLastError());
        h->launches += 1;
    }
    if (h->sorder) {
        CK(to_reference_order(h->g, h->beta, beta_out, st));
        if (c_out) CK(to_reference_order(h->g, h->c, c_out, st));
        h->launches += c_out ? 2 : 1;
    } else {
        CK(cudaMemcpyAsync(beta_out, h->beta, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
        if (c_out) CK(cudaMemcpyAsync(c_out, h->c, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    }
    cudaEventRecord(h->ev1, st);
    CK(cudaEventSynchronize(h->ev1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    S.solve_ms = ms;
    S.status = status;
    S.matvecs = h->matvecs - mv0;
    S.refinements = h->refinements - rf0;
    S.fallbacks = h->fallbacks - fb0;
    S.launches = h->launches - la0;
    if (stats) *stats = S;
    if (status == CSIPM_ERR_IPM_MAXITER) fail(h, status, "IPM reached max_iter before the tolerance");
    return status;
}

int csipm_admm(csipm_handle h, double rho, int maxt, double tol, double* z_out, csipm_admm_stats* stats) {
    if (!h || !z_out) return fail(h, CSIPM_ERR_INVALID, "null argument");
    {
        const int r = ensure_ipm_buffers(h);
        if (r) return r;
    }
    if (!(rho > 0.0) || maxt < 0) return fail(h, CSIPM_ERR_INVALID, "rho must be > 0 and maxt >= 0");
    const long long n = h->N;
    cudaStream_t st = h->stream;
    const double lam = h->lambda;
    const double* bv = h->sorder ? h->bs : h->b;
    const int ppp = passes_per_product(h->g);
    const double krylov_tol = std::sqrt(std::numeric_limits<double>::epsilon());
    csipm_admm_stats S{};
    cudaEventRecord(h->ev0, st);
    // x0 = z = ones and y = 0 in the reference packing (src/admm.jl:19-24),
    // mapped to the solve's order
    double* X[2] = {h->dba, h->db};
    double* z = h->s1;
    double* y = h->s2;
    ew_launch(fill_kernel, n, st, n, 1.0, h->sorder ? h->Qb : X[1]);
    if (h->sorder) CK(to_solver_order(h->g, h->Qb, X[1], st));
    CK(cudaMemcpyAsync(z, X[1], sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemsetAsync(y, 0, sizeof(double) * n, st));
    ew_launch(fill_kernel, n, st, n, rho, h->Db);   // A'A + rho I through the CG epilogue's diagonal
    ew_launch(admm_rhs_kernel, n, st, n, bv, z, y, rho, h->rhs);
    CK(cudaGetLastError());
    h->launches += 4;
    double err = 1.0;
    int t = 0;
    int status = CSIPM_OK;
    while (t < maxt && err > tol) {
        double* x1 = X[t & 1];
        const double* x0 = X[(t + 1) & 1];
        // x-update: Krylov cg from zero, no preconditioner, atol = rtol = sqrt(eps) (src/admm.jl:35-37)
        CK(cudaMemsetAsync(h->cgs, 0, sizeof(CgScalars), st));
        CK(cudaMemsetAsync(x1, 0, sizeof(double) * n, st));
        ew_launch(cg_init_kernel<double>, n, st, n, h->rhs, (const double*)nullptr, 0, (const double*)nullptr,
                                                        h->cg_r, h->cg_p, h->ws(h->slots + SL_DUMMY), h->cgs,
                                                        krylov_tol, krylov_tol);
        CK(cudaGetLastError());
        h->launches += 1;
        auto iteration = [&](cudaStream_t s, int it) -> cudaError_t {
            EpiCG<double> ep{h->cg_p, h->Db, h->cg_q, h->ws(&h->cgs->pq), 0.0};
            cudaError_t e = solve_AtA(h, h->cg_p, ep, &h->cgs->done, s);
            if (e != cudaSuccess) return e;
            ew_launch(cg_update_kernel<double, double>, n, s, n, it, x1, h->cg_r, h->cg_p, h->cg_q,
                                                                       (const double*)nullptr,
                                                                       h->ws(h->slots + SL_DUMMY), h->cgs);
            ew_launch(cg_pupdate_kernel<double>, n, s, n, it, h->cg_r, (const double*)nullptr, h->cg_p,
                                                               h->cgs);
            return cudaGetLastError();
        };
        {
            const int r = cg_iterations(h, &h->admm_exec[t & 1], h->opt.cg_maxit, iteration, ppp + 2);
            if (r) return r;
        }
        CK(cudaMemcpyAsync(h->hcgs, h->cgs, sizeof(CgScalars), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        S.cg_iter += h->hcgs->iters;
        h->matvecs += h->hcgs->iters;
        if (h->hcgs->breakdown) { status = fail(h, CSIPM_ERR_NONFINITE, "ADMM x-update CG breakdown"); break; }
        // z-, y-updates, the three differences and the next right-hand side
        ew_launch(admm_update_kernel, n, st, n, bv, x1, x0, z, y, rho, lam, h->rhs, h->ws(h->slots + SL_RED));
        CK(cudaGetLastError());
        h->launches += 1;
        const int r = read_slots(h, SL_RED, 3);
        if (r) return r;
        err = std::max(std::sqrt(h->hslots[SL_RED]), std::max(std::sqrt(h->hslots[SL_RED + 1]),
                                                               std::sqrt(h->hslots[SL_RED + 2])));
        if (!std::isfinite(err)) { status = fail(h, CSIPM_ERR_NONFINITE, "non-finite ADMM iterate"); break; }
        ++t;
    }
    if (h->sorder) CK(to_reference_order(h->g, z, z_out, st));
    else CK(cudaMemcpyAsync(z_out, z, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    cudaEventRecord(h->ev1, st);
    CK(cudaEventSynchronize(h->ev1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    if (status == CSIPM_OK && err > tol) status = CSIPM_ERR_IPM_MAXITER;
    S.status = status;
    S.iterations = t;
    S.err = err;
    S.solve_ms = ms;
    if (stats) *stats = S;
    return status;
}

int csipm_profile_passes(csipm_handle h, const double* x, int reps, double* ms_out, double* bytes_out,
                         char* name_out, int* npass) {
    if (!h || !x || !ms_out || !bytes_out || !npass || reps < 1) return fail(h, CSIPM_ERR_INVALID, "bad argument");
    const char* names[8];
    int np = 0, r = 0;
    // only the vectors of one CG product: D, q (and the FP32 copy of x)
    if (h->opt.precision == CSIPM_MIXED) {
        if ((!h->f_p && !h->alloc(&h->f_p, (size_t)h->N)) || (!h->f_Db && !h->alloc(&h->f_Db, (size_t)h->N)) ||
            (!h->f_q && !h->alloc(&h->f_q, (size_t)h->N)))
            return fail(h, CSIPM_ERR_OOM, h->err);
    } else if ((!h->Db && !h->alloc(&h->Db, (size_t)h->N)) || (!h->cg_q && !h->alloc(&h->cg_q, (size_t)h->N))) {
        return fail(h, CSIPM_ERR_OOM, h->err);
    }
    if (h->opt.precision == CSIPM_MIXED) {
        // the FP32 passes of the CG product, on x rounded to FP32
        ew_launch(convert_kernel<double, float>, h->N, h->stream, h->N, x, h->f_p);
        CK(cudaGetLastError());
        CK(cudaMemsetAsync(h->f_Db, 0, sizeof(float) * h->N, h->stream));
        r = profile_impl<float>(h, h->op32, h->f_p, h->f_Db, h->f_q, reps, ms_out, bytes_out, names, &np);
    } else {
        CK(cudaMemsetAsync(h->Db, 0, sizeof(double) * h->N, h->stream));
        r = profile_impl<double>(h, h->op64, x, h->Db, h->cg_q, reps, ms_out, bytes_out, names, &np);
    }
    if (r) return r;
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
