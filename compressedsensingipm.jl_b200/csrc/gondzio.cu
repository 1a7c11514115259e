// C ABI (include/csipm.h), part 5: the Gondzio formulation of the reference
// (src/gondzio_model.jl, src/gondzio_kkt.jl) as NLPModels / MadNLP-plugin
// entry points on the same handle.  beta = p - q with p, q >= 0 and a residual
// variable r: x = [p; q; r] (3N), one constraint block z0 - A(p - q) - r = 0
// (N).  The condensed Newton operator is
//     [A'A + Dp, -A'A; -A'A, A'A + Dq]
// with Dp, Dq the primal regularisation diagonals; its block preconditioner
// replaces A'A by I.  The product applies A'A once, to p - q, with the
// diagonals and the CG dot product fused into the scatter epilogue.
#include "internal.h"

namespace csipm_internal {

// obj: [0] = r.r, [1] = sum(p) + sum(q)
static __global__ void gz_obj_kernel(long long n, const double* __restrict__ x, RedWorkspace ws) {
    double acc[2] = {0.0, 0.0};
    CSIPM_GRID_LOOP(i, n) {
        const double r = x[2 * n + i];
        acc[0] += r * r;
        acc[1] += x[i] + x[n + i];
    }
    grid_reduce<2>(acc, ws, 0u, 0u);
}

static __global__ void gz_grad_kernel(long long n, const double* __restrict__ x, double lam, double* __restrict__ g) {
    CSIPM_GRID_LOOP(i, n) {
        g[i] = lam;
        g[n + i] = lam;
        g[2 * n + i] = x[2 * n + i];
    }
}

// d = a[0:n) - a[n:2n)   (sign = +1), or a[n:2n) - a[0:n) (sign = -1)
static __global__ void gz_diff_kernel(long long n, const double* __restrict__ a, double sign, double* __restrict__ d) {
    CSIPM_GRID_LOOP(i, n) d[i] = sign * (a[i] - a[n + i]);
}

// c = z0 - Ux - r
static __global__ void gz_cons_kernel(long long n, const double* __restrict__ z0, const double* __restrict__ ux,
                                      const double* __restrict__ x, double* __restrict__ c) {
    CSIPM_GRID_LOOP(i, n) c[i] = z0[i] - ux[i] - x[2 * n + i];
}

// build_kkt! (gondzio_kkt.jl:278-301)
static __global__ void gz_build_kernel(long long n, const double* __restrict__ pr_diag, double* __restrict__ Dp,
                                       double* __restrict__ Dq, double* __restrict__ P11, double* __restrict__ P12,
                                       double* __restrict__ P22) {
    CSIPM_GRID_LOOP(i, n) {
        const double rp = pr_diag[i], rq = pr_diag[n + i];
        const double ip = 1.0 / (1.0 + rp);
        const double S = 1.0 / (1.0 + rq - ip);
        P22[i] = S;
        P12[i] = ip * S;
        P11[i] = ip + ip * S * ip;
        Dp[i] = rp;
        Dq[i] = rq;
    }
}

// condensed mul! (gondzio_kkt.jl:28-53): v = (A'A (p - q))[l]
struct EpiGzMul {
    const double* x;    // 2N
    double* y;          // 2N
    const double* Dp;
    const double* Dq;
    long long n;
    double alpha, beta;
    using Pre = NoPre;
    __device__ __forceinline__ NoPre pre(int) const { return {}; }
    __device__ __forceinline__ void put(int l, double v, const NoPre&) {
        y[l] = alpha * (Dp[l] * x[l] + v) + beta * y[l];
        y[n + l] = alpha * (Dq[l] * x[n + l] - v) + beta * y[n + l];
    }
    __device__ __forceinline__ void finish() {}
};

// CG product q = K p with p.q (the PCG of solve_kkt!)
struct EpiGzCG {
    const double* p;
    double* q;
    const double* Dp;
    const double* Dq;
    long long n;
    RedWorkspace ws;
    double acc;
    struct Pre { double pp, pq, dp, dq; };
    __device__ __forceinline__ Pre pre(int l) const { return Pre{p[l], p[n + l], Dp[l], Dq[l]}; }
    __device__ __forceinline__ void put(int l, double v, const Pre& r) {
        const double a = r.dp * r.pp + v, b = r.dq * r.pq - v;
        q[l] = a;
        q[n + l] = b;
        acc += r.pp * a + r.pq * b;
    }
    __device__ __forceinline__ void finish() {
        double s[1] = {acc};
        grid_reduce<1>(s, ws, 0u, 0u);
    }
};

// kkt mul! body, first part: t = A'x_y arrives; y_p, y_q, y_r updated and d = x_q - x_p
static __global__ void gz_kktmul1_kernel(long long n, const double* __restrict__ x, const double* __restrict__ t,
                                         double* __restrict__ y, double alpha, double beta, double* __restrict__ d) {
    CSIPM_GRID_LOOP(i, n) {
        const double tv = t[i];
        y[i] = -alpha * tv + beta * y[i];
        y[n + i] = alpha * tv + beta * y[n + i];
        y[2 * n + i] = alpha * (x[2 * n + i] - x[3 * n + i]) + beta * y[2 * n + i];
        d[i] = x[n + i] - x[i];
    }
}

// second part: y_y = alpha (A d - x_r) + beta y_y
static __global__ void gz_kktmul2_kernel(long long n, const double* __restrict__ x, const double* __restrict__ ad,
                                         double* __restrict__ y, double alpha, double beta) {
    CSIPM_GRID_LOOP(i, n) y[3 * n + i] = alpha * (ad[i] - x[2 * n + i]) + beta * y[3 * n + i];
}

// jtprod!: y = [-t; t; -x]
static __global__ void gz_jtprod_kernel(long long n, const double* __restrict__ x, const double* __restrict__ t,
                                        double* __restrict__ y) {
    CSIPM_GRID_LOOP(i, n) {
        y[i] = -t[i];
        y[n + i] = t[i];
        y[2 * n + i] = -x[i];
    }
}

// solve_kkt!: buffer3 = w_r + w_y
static __global__ void gz_sum_kernel(long long n, const double* __restrict__ w, double* __restrict__ s) {
    CSIPM_GRID_LOOP(i, n) s[i] = w[2 * n + i] + w[3 * n + i];
}

// rhs = [w_p - t; w_q + t]
static __global__ void gz_rhs_kernel(long long n, const double* __restrict__ w, const double* __restrict__ t,
                                     double* __restrict__ b) {
    CSIPM_GRID_LOOP(i, n) {
        b[i] = w[i] - t[i];
        b[n + i] = w[n + i] + t[i];
    }
}

// w_x = x (and d = x_p - x_q for U dx)
static __global__ void gz_setx_kernel(long long n, const double* __restrict__ x, double* __restrict__ w,
                                      double* __restrict__ d) {
    CSIPM_GRID_LOOP(i, n) {
        const double a = x[i], b = x[n + i];
        w[i] = a;
        w[n + i] = b;
        d[i] = a - b;
    }
}

// dr = -w_y - U dx ; dy = dr - w_r(old)
static __global__ void gz_back_kernel(long long n, const double* __restrict__ udx, double* __restrict__ w) {
    CSIPM_GRID_LOOP(i, n) {
        const double wr = w[2 * n + i], wy = w[3 * n + i];
        const double dr = -wy - udx[i];
        w[2 * n + i] = dr;
        w[3 * n + i] = dr - wr;
    }
}

int ensure_gondzio_buffers(csipm_handle h) {
    int r = ensure_kkt_buffers(h);
    if (r) return r;
    if (h->gz_Dp) return CSIPM_OK;
    const size_t n = (size_t)h->N;
    if (!h->alloc(&h->gz_Dp, n) || !h->alloc(&h->gz_Dq, n) || !h->alloc(&h->gz_P11, n) || !h->alloc(&h->gz_P12, n) ||
        !h->alloc(&h->gz_P22, n) || !h->alloc(&h->gz_t1, n) || !h->alloc(&h->gz_t2, n))
        return fail(h, CSIPM_ERR_OOM, "out of device memory (Gondzio buffers)");
    return CSIPM_OK;
}

}  // namespace csipm_internal

extern "C" {

int csipm_gondzio_obj(csipm_handle h, const double* x, double* f) {
    if (!h || !x || !f) return fail(h, CSIPM_ERR_INVALID, "null argument");
    ew_launch(gz_obj_kernel, h->N, h->stream, h->N, x, h->ws(h->slots + SL_DOT));
    CK(cudaGetLastError());
    const int r = read_slots(h, SL_DOT, 2);
    if (r) return r;
    *f = 0.5 * h->hslots[SL_DOT] + h->lambda * h->hslots[SL_DOT + 1];
    return CSIPM_OK;
}

int csipm_gondzio_grad(csipm_handle h, const double* x, double* g) {
    if (!h || !x || !g) return fail(h, CSIPM_ERR_INVALID, "null argument");
    ew_launch(gz_grad_kernel, h->N, h->stream, h->N, x, h->lambda, g);
    CK(cudaGetLastError());
    return CSIPM_OK;
}

int csipm_gondzio_cons(csipm_handle h, const double* x, double* c) {
    if (!h || !x || !c) return fail(h, CSIPM_ERR_INVALID, "null argument");
    int r = ensure_gondzio_buffers(h);
    if (r) return r;
    const long long n = h->N;
    ew_launch(gz_diff_kernel, n, h->stream, n, x, 1.0, h->gz_t1);
    CK(cudaGetLastError());
    CK(op_A(h->op64, h->gz_t1, h->gz_t2, h->stream));
    ew_launch(gz_cons_kernel, n, h->stream, n, h->z0, h->gz_t2, x, c);
    CK(cudaGetLastError());
    return CSIPM_OK;
}

int csipm_gondzio_kkt_build(csipm_handle h, const double* pr_diag) {
    if (!h || !pr_diag) return fail(h, CSIPM_ERR_INVALID, "null argument");
    int r = ensure_gondzio_buffers(h);
    if (r) return r;
    ew_launch(gz_build_kernel, h->N, h->stream, h->N, pr_diag, h->gz_Dp, h->gz_Dq, h->gz_P11,
                                                                   h->gz_P12, h->gz_P22);
    CK(cudaGetLastError());
    return CSIPM_OK;
}

int csipm_gondzio_condensed_mul(csipm_handle h, double* y, const double* x, double alpha, double beta) {
    if (!h || !x || !y) return fail(h, CSIPM_ERR_INVALID, "null argument");
    if (!h->gz_Dp) return fail(h, CSIPM_ERR_INVALID, "csipm_gondzio_kkt_build must be called first");
    const long long n = h->N;
    ew_launch(gz_diff_kernel, n, h->stream, n, x, 1.0, h->gz_t1);
    CK(cudaGetLastError());
    EpiGzMul ep{x, y, h->gz_Dp, h->gz_Dq, n, alpha, beta};
    CK(op_AtA(h->op64, (const double*)h->gz_t1, ep, nullptr, h->stream));
    h->matvecs++;
    return CSIPM_OK;
}

int csipm_gondzio_precond_mul(csipm_handle h, double* y, const double* x, double alpha, double beta) {
    if (!h || !x || !y) return fail(h, CSIPM_ERR_INVALID, "null argument");
    if (!h->gz_Dp) return fail(h, CSIPM_ERR_INVALID, "csipm_gondzio_kkt_build must be called first");
    ew_launch(precond_mul_kernel, h->N, h->stream, h->N, y, x, h->gz_P11, h->gz_P12, h->gz_P22,
                                                                      alpha, beta);
    CK(cudaGetLastError());
    return CSIPM_OK;
}

int csipm_gondzio_kkt_mul(csipm_handle h, double* y, const double* x, double alpha, double beta) {
    if (!h || !x || !y) return fail(h, CSIPM_ERR_INVALID, "null argument");
    int r = ensure_gondzio_buffers(h);
    if (r) return r;
    const long long n = h->N;
    EpiStore<double> st_t{h->gz_t1};
    CK(op_At(h->op64, x + 3 * n, st_t, h->stream));
    ew_launch(gz_kktmul1_kernel, n, h->stream, n, x, h->gz_t1, y, alpha, beta, h->gz_t2);
    CK(cudaGetLastError());
    CK(op_A(h->op64, h->gz_t2, h->gz_t1, h->stream));
    ew_launch(gz_kktmul2_kernel, n, h->stream, n, x, h->gz_t1, y, alpha, beta);
    CK(cudaGetLastError());
    return CSIPM_OK;
}

int csipm_gondzio_jtprod(csipm_handle h, double* y, const double* x) {
    if (!h || !x || !y) return fail(h, CSIPM_ERR_INVALID, "null argument");
    int r = ensure_gondzio_buffers(h);
    if (r) return r;
    EpiStore<double> st_t{h->gz_t1};
    CK(op_At(h->op64, x, st_t, h->stream));
    ew_launch(gz_jtprod_kernel, h->N, h->stream, h->N, x, h->gz_t1, y);
    CK(cudaGetLastError());
    return CSIPM_OK;
}

int csipm_gondzio_kkt_solve(csipm_handle h, double* w, int* cg_iters) {
    if (!h || !w) return fail(h, CSIPM_ERR_INVALID, "null argument");
    if (!h->gz_Dp) return fail(h, CSIPM_ERR_INVALID, "csipm_gondzio_kkt_build must be called first");
    const long long n = h->N;
    cudaStream_t st = h->stream;
    const bool pc = h->opt.preconditioner != 0;
    const double *P11 = pc ? h->gz_P11 : nullptr, *P12 = pc ? h->gz_P12 : nullptr, *P22 = pc ? h->gz_P22 : nullptr;
    cudaEventRecord(h->ev0, st);
    ew_launch(gz_sum_kernel, n, st, n, w, h->gz_t1);
    EpiStore<double> st_t{h->gz_t2};
    CK(op_At(h->op64, h->gz_t1, st_t, st));
    ew_launch(gz_rhs_kernel, n, st, n, w, h->gz_t2, h->k_b);
    CK(cudaMemsetAsync(h->cgs, 0, sizeof(CgScalars), st));
    ew_launch(kcg_init_kernel, n, st, n, h->k_b, h->k_x, h->k_r, h->k_p, P11, P12, P22,
                                              h->ws(h->slots + SL_DUMMY), h->cgs, h->opt.cg_atol, h->opt.cg_rtol);
    CK(cudaGetLastError());
    int chunk = 2, since = 0;
    const int maxit = h->opt.cg_maxit;
    for (int it = 0; it < maxit; ++it) {
        ew_launch(gz_diff_kernel, n, st, n, h->k_p, 1.0, h->gz_t1);
        EpiGzCG ep{h->k_p, h->k_q, h->gz_Dp, h->gz_Dq, n, h->ws(&h->cgs->pq), 0.0};
        CK(op_AtA(h->op64, (const double*)h->gz_t1, ep, &h->cgs->done, st));
        ew_launch(kcg_update_kernel, n, st, n, it, h->k_x, h->k_r, h->k_p, h->k_q, P11, P12, P22,
                                                     h->ws(h->slots + SL_DUMMY), h->cgs);
        ew_launch(kcg_pupdate_kernel, n, st, n, it, h->k_r, h->k_p, P11, P12, P22, h->cgs);
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
    ew_launch(gz_setx_kernel, n, st, n, h->k_x, w, h->gz_t1);
    CK(cudaGetLastError());
    CK(op_A(h->op64, h->gz_t1, h->gz_t2, st));
    ew_launch(gz_back_kernel, n, st, n, h->gz_t2, w);
    CK(cudaGetLastError());
    cudaEventRecord(h->ev1, st);
    CK(cudaEventSynchronize(h->ev1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    h->krylov_ms += ms;
    if (cg_iters) *cg_iters = h->hcgs->iters;
    if (h->hcgs->breakdown) return fail(h, CSIPM_ERR_NONFINITE, "CG breakdown in the Gondzio solve_kkt");
    return CSIPM_OK;
}

}  // extern "C"
