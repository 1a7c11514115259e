// Long 1D rows: the real FFT of length N1 = 2M runs its length-M complex FFT
// as M = P*Q (four-step) over many CTAs instead of one row per CTA.
//
// Spectrum index k = k1 + P*k2 (k1 < P, k2 < Q), spatial index n = n2 + Q*n1.
// With W = exp(+2 pi i / M) for the inverse transform:
//     z[n2 + Q n1] = sum_k1 W_P^{n1 k1} W^{n2 k1} sum_k2 Z[k1 + P k2] W_Q^{n2 k2}
// and the forward transform is the same factorisation run backwards.  The
// half spectrum buffer (M+1 complex) holds every intermediate in place:
//
//   first:  lines k1 (Q values, stride P): gather beta -> X[k], X[M-k] ->
//           C2R pre-processing -> inverse DFT_Q -> twiddle conj(w_M^{n2 k1})
//           -> spec[k1 + P n2]
//   row:    rows n2 (P contiguous values): inverse DFT_P -> z[n2 + Q n1]
//           scaled and masked -> (A: store the real samples) or forward
//           DFT_P -> twiddle w_M^{n2 k1} -> spec[k1 + P n2]
//           (A^T: the row starts from the real samples instead)
//   lines:  forward DFT_Q along k2 (the ordinary strided pass)
//   post:   R2C post-processing of Z[k], Z[M-k] -> scatter to beta
//
// w_M^e = exp(-2 pi i e / M) is read from the N1-th root table (index 2e).
#pragma once
#include "operator.cuh"

namespace csipm {

// ---------------------------------------------------------------- first pass
// TB lines k1 per CTA (l1d_tiles), interleaved in shared memory as buf[x*TB + b].
template <typename T, typename TS>
__device__ __forceinline__ void l1d_first_kernel_body(PassArgs<T> a, const TS* __restrict__ src,
                                                        const cplx_t<T>* __restrict__ twN, int P, int Q, int TB) {
    using C = cplx_t<T>;
    if (a.skip && *a.skip) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* buf = reinterpret_cast<C*>(smem_raw);
    C* work = buf + Q * TB;
    __shared__ int s_rad[FFT_MAX_STAGES];
    load_radices(a.pl, s_rad);
    const int M = a.g.m1;
    const int i0 = blockIdx.x * TB;
    for (int e = threadIdx.x; e < Q * TB; e += blockDim.x) {
        const int x = e / TB, b = e % TB;
        const int k1 = i0 + b;
        C v = mk((T)0, (T)0);
        if (k1 < P) {
            const int k = k1 + P * x;
            const C xa = gather_val<T>(decode1(a.g, k), src);
            const C xb = gather_val<T>(decode1(a.g, M - k), src);
            v = c2r_pre(xa, xb, twN[k]);
        }
        buf[e] = v;
    }
    __syncthreads();
    C* res = fft_lines<T, true, true>(buf, work, s_rad, a.pl.nst, Q, TB, TB, a.tw, a.Ltab);
    for (int e = threadIdx.x; e < Q * TB; e += blockDim.x) {
        const int x = e / TB, b = e % TB;
        const int k1 = i0 + b;
        if (k1 < P) {
            C v = res[e];
            const int ex = x * k1;   // < M
            if (ex) v = cmulc(v, twN[2 * ex]);
            a.spec[k1 + (size_t)P * x] = v;
        }
    }
}
template <typename T, typename TS>
__global__ void __launch_bounds__(256) l1d_first_kernel(PassArgs<T> a, const TS* __restrict__ src,
                                                        const cplx_t<T>* __restrict__ twN, int P, int Q, int TB) {
    l1d_first_kernel_body<T, TS>(a, src, twN, P, Q, TB);
}

// ------------------------------------------------------------------ row pass
// RB rows n2 per CTA, interleaved in shared memory as buf[n1*RB + b].
template <typename T, int IN, int OUT, bool MASK>
__device__ __forceinline__ void l1d_row_kernel_body(PassArgs<T> a, const cplx_t<T>* __restrict__ twN, int P,
                                                      int Q, int RB) {
    using C = cplx_t<T>;
    if (a.skip && *a.skip) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* buf = reinterpret_cast<C*>(smem_raw);
    C* work = buf + P * RB;
    __shared__ int s_rad[FFT_MAX_STAGES];
    load_radices(a.pl, s_rad);
    const int r0 = blockIdx.x * RB;
    const int nr = min(RB, Q - r0);
    if (IN == IN_REAL) {
        // z[n] = (x[2n], x[2n+1]) with n = n2 + Q n1: consecutive rows are consecutive n
        for (int e = threadIdx.x; e < P * RB; e += blockDim.x) {
            const int b = e % RB, n1 = e / RB;
            buf[n1 * RB + b] = b < nr ? *reinterpret_cast<const C*>(a.real_in + 2 * ((size_t)(r0 + b) + (size_t)Q * n1))
                                      : mk((T)0, (T)0);
        }
    } else {
        for (int e = threadIdx.x; e < P * RB; e += blockDim.x) {
            const int b = e / P, n1 = e % P;
            buf[n1 * RB + b] = b < nr ? a.spec[(size_t)P * (r0 + b) + n1] : mk((T)0, (T)0);
        }
    }
    __syncthreads();
    C* c1 = buf;
    C* other = work;
    if (IN != IN_REAL) {
        c1 = fft_lines<T, true, true>(buf, work, s_rad, a.pl.nst, P, RB, RB, a.tw, a.Ltab);
        other = (c1 == buf) ? work : buf;
    }
    const T sc = (T)a.scale;
    for (int e = threadIdx.x; e < P * RB; e += blockDim.x) {
        const int b = e % RB, n1 = e / RB;
        if (b < nr) {
            const size_t n = (size_t)(r0 + b) + (size_t)Q * n1;
            C y = c1[n1 * RB + b];
            y.x *= sc;
            y.y *= sc;
            if (MASK) {
                const uint32_t w = a.maskw[n >> 4];
                const int sh = (int)((2 * n) & 31);
                if (!((w >> sh) & 1u)) y.x = (T)0;
                if (!((w >> (sh + 1)) & 1u)) y.y = (T)0;
            }
            if (OUT == OUT_REAL) *reinterpret_cast<C*>(a.real_out + 2 * n) = y;
            else c1[n1 * RB + b] = y;
        }
    }
    if (OUT == OUT_REAL) return;
    __syncthreads();
    C* c2 = fft_lines<T, false, true>(c1, other, s_rad, a.pl.nst, P, RB, RB, a.tw, a.Ltab);
    for (int e = threadIdx.x; e < P * RB; e += blockDim.x) {
        const int b = e / P, k1 = e % P;
        if (b < nr) {
            const int n2 = r0 + b;
            C v = c2[k1 * RB + b];
            const int ex = n2 * k1;   // < M
            if (ex) v = cmul(v, twN[2 * ex]);
            a.spec[(size_t)P * n2 + k1] = v;
        }
    }
}
template <typename T, int IN, int OUT, bool MASK>
__global__ void __launch_bounds__(256) l1d_row_kernel(PassArgs<T> a, const cplx_t<T>* __restrict__ twN, int P,
                                                      int Q, int RB) {
    l1d_row_kernel_body<T, IN, OUT, MASK>(a, twN, P, Q, RB);
}

// ------------------------------------------------------------------ post pass
// X[k] from Z[k], Z[M-k] (k = 0 also gives X[M]) and the scatter to beta.
template <typename T, class Epi>
__device__ __forceinline__ void l1d_post_kernel_body(PassArgs<T> a, const cplx_t<T>* __restrict__ twN, Epi epi) {
    using C = cplx_t<T>;
    if (a.skip && *a.skip) return;
    const int M = a.g.m1;
    const int half = M / 2;
    Epi ep = epi;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k <= half; k += gridDim.x * blockDim.x) {
        if (k == 0) {
            const C z0 = a.spec[0];
            scatter_one<T>(decode1(a.g, 0), r2c_post(z0, z0, twN[0]), ep);
            scatter_one<T>(decode1(a.g, M), mk((T)2 * (z0.x - z0.y), (T)0), ep);
        } else if (2 * k == M) {
            const C zk = a.spec[k];
            scatter_one<T>(decode1(a.g, k), r2c_post(zk, zk, twN[k]), ep);
        } else {
            const C zk = a.spec[k], zm = a.spec[M - k];
            scatter_one<T>(decode1(a.g, k), r2c_post(zk, zm, twN[k]), ep);
            scatter_one<T>(decode1(a.g, M - k), r2c_post(zm, zk, twN[M - k]), ep);
        }
    }
    ep.finish();
}
template <typename T, class Epi>
__global__ void __launch_bounds__(256) l1d_post_kernel(PassArgs<T> a, const cplx_t<T>* __restrict__ twN, Epi epi) {
    l1d_post_kernel_body<T, Epi>(a, twN, epi);
}

}  // namespace csipm

namespace csipm {

// ---------------------------------------------------------------- launchers
template <typename T>
PassArgs<T> l1d_args(const FftOperator<T>& op, bool row, double scale, const int* skip) {
    PassArgs<T> a{};
    a.g = op.g;
    a.spec = op.spec;
    a.pl = row ? op.planP : op.planQ;
    a.tw = row ? op.twP : op.twQ;
    a.Ltab = row ? op.l1P : op.l1Q;
    a.maskw = op.maskw;
    a.wpr = op.wpr;
    a.scale = scale;
    a.skip = skip;
    return a;
}

template <typename T, typename TS>
cudaError_t l1d_first(const FftOperator<T>& op, const TS* src, const int* skip, cudaStream_t st) {
    auto k = l1d_first_kernel<T, TS>;
    const size_t smem = 2 * (size_t)op.l1Q * op.l1TB * sizeof(cplx_t<T>);
    cudaError_t e = smem_optin(k, smem);
    if (e != cudaSuccess) return e;
    k<<<(op.l1P + op.l1TB - 1) / op.l1TB, 256, smem, st>>>(l1d_args(op, false, 1.0, skip), src, op.tw1, op.l1P,
                                                            op.l1Q, op.l1TB);
    return cudaGetLastError();
}

template <typename T, int IN, int OUT, bool MASK>
cudaError_t l1d_row(const FftOperator<T>& op, double scale, const T* real_in, T* real_out, const int* skip,
                    cudaStream_t st) {
    auto k = l1d_row_kernel<T, IN, OUT, MASK>;
    const size_t smem = 2 * (size_t)op.l1P * op.l1RB * sizeof(cplx_t<T>);
    cudaError_t e = smem_optin(k, smem);
    if (e != cudaSuccess) return e;
    PassArgs<T> a = l1d_args(op, true, scale, skip);
    a.real_in = real_in;
    a.real_out = real_out;
    k<<<(op.l1Q + op.l1RB - 1) / op.l1RB, 256, smem, st>>>(a, op.tw1, op.l1P, op.l1Q, op.l1RB);
    return cudaGetLastError();
}

template <typename T>
cudaError_t l1d_lines_forward(const FftOperator<T>& op, const int* skip, cudaStream_t st) {
    PassArgs<T> a = l1d_args(op, false, 1.0, skip);
    a.tw_in_smem = op.q_cfg.tw_in_smem;
    a.n_lines = op.l1P;
    a.n_outer = 1;
    a.so = 0;
    a.sx = op.l1P;
    a.jk_mode = 2;
    EpiStore<double> none{nullptr};
    return launch_strided<T, false, IN_SPEC, OUT_SPEC>(op.q_cfg, a, (const double*)nullptr, none, st);
}

template <typename T, class Epi>
cudaError_t l1d_post(const FftOperator<T>& op, const Epi& epi, const int* skip, cudaStream_t st) {
    const int half = op.g.m1 / 2 + 1;
    int blocks = (half + 255) / 256;
    if (blocks > 1024) blocks = 1024;
    l1d_post_kernel<T, Epi><<<blocks, 256, 0, st>>>(l1d_args(op, false, 1.0, skip), op.tw1, epi);
    return cudaGetLastError();
}

}  // namespace csipm
