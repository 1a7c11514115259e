// C ABI (include/csipm.h), part 2: the NLPModels (src/fft_model.jl) and
// MadNLP KKT-plugin (src/fft_kkt.jl) entry points.
#include "internal.h"

namespace csipm_internal {

int ensure_kkt_buffers(csipm_handle h) {
    if (h->L1) return CSIPM_OK;
    const size_t n = (size_t)h->N;
    if (!h->alloc(&h->L1, n) || !h->alloc(&h->L2, n) || !h->alloc(&h->P11, n) || !h->alloc(&h->P12, n) ||
        !h->alloc(&h->P22, n) || !h->alloc(&h->k_b, 2 * n) || !h->alloc(&h->k_x, 2 * n) || !h->alloc(&h->k_r, 2 * n) ||
        !h->alloc(&h->k_p, 2 * n) || !h->alloc(&h->k_q, 2 * n))
        return fail(h, CSIPM_ERR_OOM, "out of device memory (KKT buffers)");
    return CSIPM_OK;
}

}  // namespace csipm_internal

extern "C" {

int csipm_obj(csipm_handle h, const double* x, double* f) {
    if (!h || !x || !f) return fail(h, CSIPM_ERR_INVALID, "null argument");
    // 1/2 ||A beta||^2 = 1/2 beta' A'A beta (P is a projection); - beta'A^T z0 ; + lambda sum(c)
    EpiStore<double> ep{h->Qb};
    CK(op_AtA(h->op64, x, ep, nullptr, h->stream));
    h->matvecs++;
    const long long n = h->N;
    ew_launch(dot2_kernel, n, h->stream, n, x, h->Qb, x, h->b, h->ws(h->slots + SL_DOT));
    CK(cudaGetLastError());
    // sum(c) = c . 1 : reuse Minv as a ones vector would cost a fill; use a dedicated reduction
    ew_launch(fill_kernel, n, h->stream, n, 1.0, h->rhs);
    ew_launch(dot2_kernel, n, h->stream, n, x + n, h->rhs, nullptr, nullptr, h->ws(h->slots + SL_DOT + 2));
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
    ew_launch(fill_kernel, h->N, h->stream, h->N, h->lambda, g + h->N);
    CK(cudaGetLastError());
    return CSIPM_OK;
}

int csipm_cons(csipm_handle h, const double* x, double* c) {
    if (!h || !x || !c) return fail(h, CSIPM_ERR_INVALID, "null argument");
    ew_launch(cons_kernel, h->N, h->stream, h->N, x, c);
    CK(cudaGetLastError());
    return CSIPM_OK;
}

int csipm_hprod(csipm_handle h, const double* v, double* hv, double obj_weight) {
    if (!h || !v || !hv) return fail(h, CSIPM_ERR_INVALID, "null argument");
    EpiScale ep{obj_weight, hv};
    CK(op_AtA(h->op64, v, ep, nullptr, h->stream));
    h->matvecs++;
    ew_launch(fill_kernel, h->N, h->stream, h->N, 0.0, hv + h->N);
    CK(cudaGetLastError());
    return CSIPM_OK;
}

int csipm_kkt_build(csipm_handle h, const double* pr_diag) {
    if (!h || !pr_diag) return fail(h, CSIPM_ERR_INVALID, "null argument");
    int r = ensure_kkt_buffers(h);
    if (r) return r;
    ew_launch(kkt_build_kernel, h->N, h->stream, h->N, pr_diag, h->L1, h->L2, h->P11, h->P12, h->P22);
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
    ew_launch(precond_mul_kernel, h->N, h->stream, h->N, y, x, h->P11, h->P12, h->P22, alpha, beta);
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
    ew_launch(jtprod_kernel, h->N, h->stream, h->N, y, x);
    CK(cudaGetLastError());
    return CSIPM_OK;
}

int csipm_kkt_solve(csipm_handle h, double* w, const double* pr_diag, int* cg_iters) {
    if (!h || !w || !pr_diag) return fail(h, CSIPM_ERR_INVALID, "null argument");
    if (!h->L1) return fail(h, CSIPM_ERR_INVALID, "csipm_kkt_build must be called first");
    const long long n = h->N;
    cudaStream_t st = h->stream;
    const bool pc = h->opt.preconditioner != 0;
    const double *P11 = pc ? h->P11 : nullptr, *P12 = pc ? h->P12 : nullptr, *P22 = pc ? h->P22 : nullptr;
    cudaEventRecord(h->ev0, st);
    ew_launch(kkt_rhs_kernel, n, st, n, w, pr_diag, h->k_b);
    CK(cudaMemsetAsync(h->cgs, 0, sizeof(CgScalars), st));
    ew_launch(kcg_init_kernel, n, st, n, h->k_b, h->k_x, h->k_r, h->k_p, P11, P12, P22,
                                              h->ws(h->slots + SL_DUMMY), h->cgs, h->opt.cg_atol, h->opt.cg_rtol);
    CK(cudaGetLastError());
    int chunk = 2, since = 0;
    const int maxit = h->opt.cg_maxit;
    for (int it = 0; it < maxit; ++it) {
        EpiKcg ep{h->k_p, h->k_q, h->L1, h->L2, n, h->ws(&h->cgs->pq), 0.0};
        CK(op_AtA(h->op64, h->k_p, ep, &h->cgs->done, st));
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
    ew_launch(kkt_back_kernel, n, st, n, w, h->k_x, pr_diag);
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

}  // extern "C"
