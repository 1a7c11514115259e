// A^T A without any device allocation: csipm_apply_AtA_static.
//
// Some callers cannot call cudaMalloc: code that runs inside a runtime owning
// all device memory through its own pool (a Julia CUDA.jl or PyTorch process
// with a hard memory limit, a serving process that pre-commits the whole HBM
// to resident problems), and latency-critical loops that cannot afford the
// implicit device synchronisation of cudaMalloc/cudaFree.  For them this file
// keeps the operator's only scratch — the half spectrum and the twiddle tables
// — in one file-scope device array of fixed size.  Every GPU that loads the
// library holds the array until the process exits; all calls share it, so
// calls that overlap on the GPU race, and each call rewrites everything it
// reads: a small kernel writes the twiddle tables for the call's sizes (no
// host-to-device copy) and the first pass writes the whole spectrum.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/csipm.h"
#include "geometry.h"
#include "long1d.cuh"
#include "operator.cuh"

using namespace csipm;

namespace csipm {
void set_last_error(const std::string& msg);   // api.cu
}

namespace {

constexpr size_t STATIC_SCRATCH_BYTES = (size_t)32 << 20;   // 32 MiB

static __device__ __align__(256) unsigned char g_static_scratch[STATIC_SCRATCH_BYTES];

constexpr int MAX_DEVICES = 64;
std::mutex g_setup_mu;
void* g_scratch_addr[MAX_DEVICES] = {nullptr};

int static_fail(int status, const std::string& msg) {
    set_last_error(msg);   // reported by csipm_last_error(NULL)
    return status;
}

// Device address of the scratch array on the current device (looked up once
// per device, with that device current; the host-side symbol is only a stand-in).
int scratch_address(void** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return static_fail(CSIPM_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= MAX_DEVICES) return static_fail(CSIPM_ERR_UNSUPPORTED, "device index out of range");
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess) return static_fail(CSIPM_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return CSIPM_OK;
}

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// twiddle tables: the handle path's device-built tables (launch_twiddles),
// so both entry points apply the same operator bit for bit
cudaError_t put_twiddles(int L, double2* dst, cudaStream_t st) { return launch_twiddles(L, dst, st); }

}  // namespace

extern "C" {

int csipm_apply_AtA_static(int dim, const int* size, const uint32_t* keep_bits, const double* x, double* y,
                           void* stream) {
    if (dim < 1 || dim > 3 || !size) return static_fail(CSIPM_ERR_INVALID, "dim must be 1, 2 or 3");
    if (!x || !y) return static_fail(CSIPM_ERR_INVALID, "x and y must be device pointers");
    for (int d = 0; d < dim; ++d)
        if (size[d] < 2 || size[d] % 2) return static_fail(CSIPM_ERR_ODD_DIM, "every dimension must be even and >= 2");
    int n[3] = {size[0], dim >= 2 ? size[1] : 1, dim >= 3 ? size[2] : 1};
    if ((long long)n[0] * n[1] * n[2] >= (1LL << 31)) return static_fail(CSIPM_ERR_UNSUPPORTED, "N must be below 2^31");
    const Geom g = make_geom(dim, n, n[0] / 2 + 1);
    using C = double2;

    // operator description over the static scratch (no allocation anywhere):
    // plans and pass configurations first, then the carve-up of the array
    FftOperator<double> op;
    op.owns = false;
    op.g = g;
    op.stream = (cudaStream_t)stream;
    std::string err;
    const bool long1d = dim == 1 && g.m1 > L1D_MIN_M;   // the handle path's four-step rows
    if (long1d) {
        if (!l1d_split(g.m1, &op.l1P, &op.l1Q))
            return static_fail(CSIPM_ERR_UNSUPPORTED, "1D length has no split M = P*Q with P <= 4096, Q <= 768");
        if (!make_fft_plan(op.l1P, &op.planP, &err, op.max_radix()) ||
            !make_fft_plan(op.l1Q, &op.planQ, &err, op.max_radix()))
            return static_fail(CSIPM_ERR_UNSUPPORTED, err);
        if (!op.choose_strided(op.planQ, op.l1Q, op.l1P, 1, &op.q_cfg, &err)) return static_fail(CSIPM_ERR_UNSUPPORTED, err);
        l1d_tiles(op.l1P, op.l1Q, sizeof(C), &op.l1TB, &op.l1RB);
        op.plan1 = op.planP;
    } else {
        if (!op.make_plans(&err)) return static_fail(CSIPM_ERR_UNSUPPORTED, err);
        if (!op.choose_row(g.n2 * g.n3, &op.row_cfg, &err)) return static_fail(CSIPM_ERR_UNSUPPORTED, err);
    }
    if (dim >= 2 && !op.choose_strided(op.plan2, g.n2, g.m1 + 1, dim == 3 ? g.n3 : 1, &op.s2_cfg, &err))
        return static_fail(CSIPM_ERR_UNSUPPORTED, err);
    if (dim >= 3 && !op.choose_strided(op.plan3, g.n3, g.m1 + 1, g.n2, &op.s3_cfg, &err))
        return static_fail(CSIPM_ERR_UNSUPPORTED, err);

    const size_t spec_b = align256(sizeof(C) * (size_t)g.ld1 * g.n2 * g.n3);
    const size_t tw1_b = align256(sizeof(C) * (size_t)g.n1);
    const size_t tw2_b = dim >= 2 ? align256(sizeof(C) * (size_t)g.n2) : 0;
    const size_t tw3_b = dim >= 3 ? align256(sizeof(C) * (size_t)g.n3) : 0;
    const size_t twP_b = long1d ? align256(sizeof(C) * (size_t)op.l1P) : 0;
    const size_t twQ_b = long1d ? align256(sizeof(C) * (size_t)op.l1Q) : 0;
    const size_t need = spec_b + tw1_b + tw2_b + tw3_b + twP_b + twQ_b;
    if (need > STATIC_SCRATCH_BYTES)
        return static_fail(CSIPM_ERR_UNSUPPORTED, "problem needs " + std::to_string(need) +
                                                      " bytes of scratch; csipm_apply_AtA_static holds at most " +
                                                      std::to_string(STATIC_SCRATCH_BYTES) + " bytes (32 MiB)");
    void* base = nullptr;
    int st = scratch_address(&base);
    if (st) return st;
    unsigned char* p = static_cast<unsigned char*>(base);
    size_t off = 0;
    auto carve = [&](size_t b) { C* q = b ? reinterpret_cast<C*>(p + off) : nullptr; off += b; return q; };
    op.spec = carve(spec_b);
    op.tw1 = carve(tw1_b);
    op.tw2 = carve(tw2_b);
    op.tw3 = carve(tw3_b);
    op.twP = carve(twP_b);
    op.twQ = carve(twQ_b);
    op.maskw = const_cast<uint32_t*>(keep_bits);   // read-only in every pass
    op.wpr = (g.n1 + 31) / 32;

    // twiddle tables of this call's sizes (the array keeps the last call's contents)
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = put_twiddles(g.n1, op.tw1, s);
    if (e == cudaSuccess && dim >= 2) e = put_twiddles(g.n2, op.tw2, s);
    if (e == cudaSuccess && dim >= 3) e = put_twiddles(g.n3, op.tw3, s);
    if (e == cudaSuccess && long1d) e = put_twiddles(op.l1P, op.twP, s);
    if (e == cudaSuccess && long1d) e = put_twiddles(op.l1Q, op.twQ, s);
    if (e != cudaSuccess) return static_fail(CSIPM_ERR_CUDA, std::string("twiddle kernel: ") + cudaGetErrorString(e));

    // the fused passes of A^T A: five (3D), three (2D), one row pass (1D) or
    // the four passes of a long 1D row
    const double sc = 1.0 / (2.0 * (double)g.N);
    const bool mask = keep_bits != nullptr;
    EpiStore<double> none{nullptr};
    EpiStore<double> out{y};
    PassArgs<double> ra = op.row_args(sc, nullptr, nullptr);
    if (long1d) {
        e = l1d_first(op, x, nullptr, s);
        if (e == cudaSuccess)
            e = mask ? l1d_row<double, IN_SPEC, OUT_SPEC, true>(op, sc, nullptr, nullptr, nullptr, s)
                     : l1d_row<double, IN_SPEC, OUT_SPEC, false>(op, sc, nullptr, nullptr, nullptr, s);
        if (e == cudaSuccess) e = l1d_lines_forward(op, nullptr, s);
        if (e == cudaSuccess) e = l1d_post(op, out, nullptr, s);
    } else if (dim == 1) {
        e = mask ? launch_row<double, IN_GATHER, OUT_SCATTER, true>(op.row_cfg, ra, x, out, s)
                 : launch_row<double, IN_GATHER, OUT_SCATTER, false>(op.row_cfg, ra, x, out, s);
    } else {
        // beta-side passes along dim 2, plain spectrum passes along dim 3
        PassArgs<double> a2 = op.strided_args(2);
        PassArgs<double> a3 = dim == 3 ? op.strided_args(3) : a2;
        e = launch_strided<double, true, IN_GATHER, OUT_SPEC>(op.s2_cfg, a2, x, none, s);
        if (e == cudaSuccess && dim == 3)
            e = launch_strided<double, true, IN_SPEC, OUT_SPEC>(op.s3_cfg, a3, (const double*)nullptr, none, s);
        if (e == cudaSuccess)
            e = mask ? launch_row<double, IN_SPEC, OUT_SPEC, true>(op.row_cfg, ra, (const double*)nullptr, none, s)
                     : launch_row<double, IN_SPEC, OUT_SPEC, false>(op.row_cfg, ra, (const double*)nullptr, none, s);
        if (e == cudaSuccess && dim == 3)
            e = launch_strided<double, false, IN_SPEC, OUT_SPEC>(op.s3_cfg, a3, (const double*)nullptr, none, s);
        if (e == cudaSuccess)
            e = launch_strided<double, false, IN_SPEC, OUT_SCATTER>(op.s2_cfg, a2, (const double*)nullptr, out, s);
    }
    if (e != cudaSuccess) return static_fail(CSIPM_ERR_CUDA, std::string("CUDA: ") + cudaGetErrorString(e));
    return CSIPM_OK;
}

}  // extern "C"
