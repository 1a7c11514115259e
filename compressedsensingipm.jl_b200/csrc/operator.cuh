// The masked sampling operator A = P_Omega * sqrt(N) * Re(IDFT(B .)) and its
// adjoint, applied matrix-free through fused real-FFT passes.
//
// Layout in HBM: one half spectrum (M1+1) x N2 x N3 of complex values, dim 1
// fastest, pitch ld1; the mask as one bit per real sample, rows of N1 bits
// padded to 32-bit words.  Pass structure (3D; 2D drops the dim-3 passes, 1D is
// a single row pass):
//
//   A^T A x :  [gather x -> inverse FFT dim 3] -> [inverse dim 2]
//              -> [row: C2R dim 1, scale, mask, R2C dim 1]
//              -> [forward dim 2] -> [forward dim 3 -> scatter + epilogue]
//
// The beta -> spectrum gather is fused into the first pass and the
// spectrum -> beta scatter (plus any elementwise epilogue, e.g. the CG's
// q = A^T A p + D p and p.q) into the last, so beta-space vectors are touched
// once per product and the real-space samples never reach HBM.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>
#include <set>
#include <string>
#include <utility>
#include <vector>

#include "cplx.cuh"
#include "fft_device.cuh"
#include "geometry.h"
#include "plan.h"
#include "reduce.cuh"

namespace csipm {

// *_SGATHER / *_SSCATTER: beta-space vectors in solver order (geometry.h)
enum PassIn { IN_SPEC = 0, IN_GATHER = 1, IN_REAL = 2, IN_SGATHER = 3 };
enum PassOut { OUT_SPEC = 0, OUT_SCATTER = 1, OUT_REAL = 2, OUT_SSCATTER = 3 };

constexpr double SQRT2_D = 1.4142135623730951;

template <typename T>
struct PassArgs {
    Geom g;
    FftPlanDev pl;
    const cplx_t<T>* tw;     // Ltab-th roots of unity (global memory)
    int Ltab;
    int tw_in_smem;
    cplx_t<T>* spec;
    // strided passes
    int n_lines;             // number of dim-1 positions (M1+1)
    int n_outer;             // number of lines per dim-1 position (outer index range)
    long long so, sx;        // element strides of the outer index and of the transform index
    int jk_mode;             // 0: (j,k) = (o,x)   1: (j,k) = (x,o)   2: (j,k) = (x,0)
    // row passes
    int nrows, rb, tbp;
    const uint32_t* maskw;
    int wpr;
    double scale;
    const T* real_in;
    T* real_out;
    const int* skip;         // when non-null and *skip != 0 the pass returns at once (converged CG)
    const int4* pmap;        // solver order: (re, im, kind, src) of the planes i = 0, M1, index (p*N3 + k)*N2 + j
};

// ------------------------------------------------------------- async copies
// cp.async (LDGSTS): global -> shared without register staging, many in flight
// per thread; completion is waited for with cp.async.wait_group (never spins).
__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

template <int BYTES> __device__ __forceinline__ void cp_async(void* s, const void* g);
template <> __device__ __forceinline__ void cp_async<16>(void* s, const void* g) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_addr(s)), "l"(g) : "memory");
}
template <> __device__ __forceinline__ void cp_async<8>(void* s, const void* g) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem_addr(s)), "l"(g) : "memory");
}
template <> __device__ __forceinline__ void cp_async<4>(void* s, const void* g) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(smem_addr(s)), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// ------------------------------------------------------------- epilogues
// Two-phase epilogues: pre(l) loads what put(l, v, pre) needs, so a scatter
// loop can issue the loads of several elements before it consumes them.
struct NoPre {};

// pre2 / put2 act on the solver-order pair l (elements 2l, 2l+1) with one
// vector access per operand.
template <typename TO>
struct EpiStore {
    TO* out;
    using Pre = NoPre;
    using Pre2 = NoPre;
    __device__ __forceinline__ NoPre pre(int) const { return {}; }
    __device__ __forceinline__ void put(int l, double v, const NoPre&) { out[l] = (TO)v; }
    __device__ __forceinline__ NoPre pre2(int64_t) const { return {}; }
    __device__ __forceinline__ void put2(int64_t l, double x, double y, const NoPre&) {
        reinterpret_cast<cplx_t<TO>*>(out)[l] = mk((TO)x, (TO)y);
    }
    __device__ __forceinline__ void finish() {}
};

// q = A^T A p + D .* p, accumulating p.q (CG product)
template <typename TV>
struct EpiCG {
    const TV* p;
    const TV* D;
    TV* q;
    RedWorkspace ws;
    double acc;
    struct Pre { double p, d; };
    struct Pre2 { cplx_t<TV> p, d; };
    __device__ __forceinline__ Pre pre(int l) const { return Pre{(double)p[l], (double)D[l]}; }
    __device__ __forceinline__ void put(int l, double v, const Pre& r) {
        const TV qv = (TV)(v + r.d * r.p);
        q[l] = qv;
        acc += r.p * (double)qv;
    }
    __device__ __forceinline__ Pre2 pre2(int64_t l) const {
        return Pre2{reinterpret_cast<const cplx_t<TV>*>(p)[l], reinterpret_cast<const cplx_t<TV>*>(D)[l]};
    }
    __device__ __forceinline__ void put2(int64_t l, TV x, TV y, const Pre2& r) {
        const TV qx = x + r.d.x * r.p.x;
        const TV qy = y + r.d.y * r.p.y;
        reinterpret_cast<cplx_t<TV>*>(q)[l] = mk(qx, qy);
        acc += (double)r.p.x * (double)qx + (double)r.p.y * (double)qy;
    }
    __device__ __forceinline__ void finish() {
        double a[1] = {acc};
        grid_reduce<1>(a, ws, 0u, 0u);
    }
};

// ------------------------------------------------------- gather / scatter
template <typename T, typename TS>
__device__ __forceinline__ cplx_t<T> gather_val(const MapEntry& e, const TS* __restrict__ src) {
    if (e.kind == KIND_VERT) return mk((T)src[e.re], (T)0);
    const T r = (T)0.7071067811865476;   // 1/sqrt(2) (the operator is tolerance-checked, not bitwise)
    const T a = (T)src[e.re], b = (T)src[e.im];
    return e.kind == KIND_PLUS ? mk(a * r, b * r) : mk(a * r, -b * r);
}

// staged (re, im) of beta -> spectrum value, in place
template <typename T>
__device__ __forceinline__ cplx_t<T> gather_combine(const MapEntry& e, cplx_t<T> v) {
    const T r = (T)0.7071067811865476;
    if (e.kind == KIND_VERT) return mk(v.x, (T)0);
    return e.kind == KIND_PLUS ? mk(v.x * r, v.y * r) : mk(v.x * r, -v.y * r);
}

// start the async copies of the two beta values of a spectrum position into its slot
template <typename T, typename TS>
__device__ __forceinline__ void gather_issue(const MapEntry& e, const TS* __restrict__ src, cplx_t<T>* slot) {
    if constexpr (sizeof(TS) == sizeof(T)) {
        cp_async<sizeof(TS)>(&slot->x, src + e.re);
        if (e.kind != KIND_VERT) cp_async<sizeof(TS)>(&slot->y, src + e.im);
        else slot->y = (T)0;
    } else {   // precisions differ: plain loads (no pass gathers this way; kept for completeness)
        slot->x = (T)src[e.re];
        slot->y = e.kind != KIND_VERT ? (T)src[e.im] : (T)0;
    }
}

template <typename T, class Epi>
__device__ __forceinline__ void scatter_one(const MapEntry& e, cplx_t<T> v, Epi& ep) {
    if (!e.src) return;
    const typename Epi::Pre pr = ep.pre(e.re);
    if (e.kind == KIND_VERT) {
        ep.put(e.re, (double)v.x, pr);
    } else {
        const typename Epi::Pre pi = ep.pre(e.im);
        ep.put(e.re, SQRT2_D * (double)v.x, pr);
        ep.put(e.im, (e.kind == KIND_PLUS ? SQRT2_D : -SQRT2_D) * (double)v.y, pi);
    }
}

// Scatter a tile held in shared memory: element e (= smem index) maps to the
// spectrum position coord(e) -> (ok, i, j, k).  U elements per thread are
// decoded and their epilogue operands loaded before any is consumed.
template <typename T, int U, class Epi, class Coord>
__device__ __forceinline__ void scatter_tile(const cplx_t<T>* res, int total, const Geom& g, Coord coord, Epi& ep) {
    for (int e0 = threadIdx.x; e0 < total; e0 += U * blockDim.x) {
        MapEntry en[U];
        typename Epi::Pre pr[U], pi[U];
        bool ok[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int e = e0 + u * blockDim.x;
            int i = 0, j = 0, k = 0;
            ok[u] = (e < total) && coord(e, i, j, k);
            if (ok[u]) {
                en[u] = decode(g, i, j, k);
                ok[u] = en[u].src != 0;
            }
            if (ok[u]) {
                pr[u] = ep.pre(en[u].re);
                if (en[u].kind != KIND_VERT) pi[u] = ep.pre(en[u].im);
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (!ok[u]) continue;
            const cplx_t<T> v = res[e0 + u * blockDim.x];
            if (en[u].kind == KIND_VERT) {
                ep.put(en[u].re, (double)v.x, pr[u]);
            } else {
                ep.put(en[u].re, SQRT2_D * (double)v.x, pr[u]);
                ep.put(en[u].im, (en[u].kind == KIND_PLUS ? SQRT2_D : -SQRT2_D) * (double)v.y, pi[u]);
            }
        }
    }
}

__device__ __forceinline__ void jk_of(int mode, int o, int x, int& j, int& k) {
    if (mode == 0) { j = o; k = x; }
    else if (mode == 1) { j = x; k = o; }
    else { j = x; k = 0; }
}

constexpr int SCATTER_UNROLL = 4;

// ------------------------------------------------------------ strided pass
// Persistent: each CTA walks tiles t = blockIdx.x, blockIdx.x + gridDim.x, ...
// A tile is TB consecutive dim-1 positions x one full line along the axis.
// Shared memory: two load buffers (the next tile streams in by cp.async while
// the current one is transformed) and one work buffer for the ping-pong stages.
template <typename T, int TB, bool INV, int IN, int OUT, typename TS, class Epi>
__device__ __forceinline__ void strided_pass_kernel_body(PassArgs<T> a, const TS* __restrict__ src, Epi epi) {
    using C = cplx_t<T>;
    if (a.skip && *a.skip) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int L = a.pl.L;
    const int Lb = L * TB;
    C* buf0 = reinterpret_cast<C*>(smem_raw);
    C* buf1 = buf0 + Lb;
    C* work = buf1 + Lb;
    __shared__ int s_rad[FFT_MAX_STAGES];
    load_radices(a.pl, s_rad);
    const C* tw = a.tw;
    if (a.tw_in_smem) {
        C* tws = work + Lb;
        for (int e = threadIdx.x; e < a.Ltab; e += blockDim.x) tws[e] = a.tw[e];
        tw = tws;
    }
    const int tiles_x = (a.n_lines + TB - 1) / TB;
    const int ntiles = tiles_x * a.n_outer;
    const C zero = mk((T)0, (T)0);

    auto issue = [&](int t, C* dst) {
        const int tx = t % tiles_x, o = t / tiles_x;
        const int i0 = tx * TB, nb = min(TB, a.n_lines - i0);
        const long long base = i0 + (long long)o * a.so;
        for (int e = threadIdx.x; e < Lb; e += blockDim.x) {
            const int x = e / TB, b = e % TB;
            if (b < nb) {
                if (IN == IN_SPEC) {
                    cp_async<sizeof(C)>(&dst[e], a.spec + base + b + (long long)x * a.sx);
                } else {
                    int j, k;
                    jk_of(a.jk_mode, o, x, j, k);
                    gather_issue<T>(decode(a.g, i0 + b, j, k), src, &dst[e]);
                }
            } else {
                dst[e] = zero;
            }
        }
    };

    Epi ep = epi;
    int t = blockIdx.x;
    if (t < ntiles) issue(t, buf0);
    cp_async_commit();
    for (int it = 0; t < ntiles; t += gridDim.x, ++it) {
        C* cur = (it & 1) ? buf1 : buf0;
        C* nxt = (it & 1) ? buf0 : buf1;
        if (t + (int)gridDim.x < ntiles) issue(t + gridDim.x, nxt);
        cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
        const int tx = t % tiles_x, o = t / tiles_x;
        const int i0 = tx * TB, nb = min(TB, a.n_lines - i0);
        if (IN == IN_GATHER) {
            for (int e = threadIdx.x; e < Lb; e += blockDim.x) {
                const int x = e / TB, b = e % TB;
                if (b < nb) {
                    int j, k;
                    jk_of(a.jk_mode, o, x, j, k);
                    cur[e] = gather_combine<T>(decode(a.g, i0 + b, j, k), cur[e]);
                }
            }
            __syncthreads();
        }
        const C* res = fft_lines<T, INV, true>(cur, work, s_rad, a.pl.nst, L, TB, TB, tw, a.Ltab);
        if (OUT == OUT_SPEC) {
            const long long base = i0 + (long long)o * a.so;
            for (int e = threadIdx.x; e < Lb; e += blockDim.x) {
                const int x = e / TB, b = e % TB;
                if (b < nb) a.spec[base + b + (long long)x * a.sx] = res[e];
            }
        } else {
            const int mode = a.jk_mode;
            auto coord = [&](int e, int& i, int& j, int& k) -> bool {
                const int x = e / TB, b = e % TB;
                if (b >= nb) return false;
                i = i0 + b;
                jk_of(mode, o, x, j, k);
                return true;
            };
            scatter_tile<T, SCATTER_UNROLL>(res, Lb, a.g, coord, ep);
        }
        __syncthreads();
    }
    if (OUT == OUT_SCATTER) ep.finish();
}
template <typename T, int TB, bool INV, int IN, int OUT, typename TS, class Epi>
__global__ void __launch_bounds__(256) strided_pass_kernel(PassArgs<T> a, const TS* __restrict__ src, Epi epi) {
    strided_pass_kernel_body<T, TB, INV, IN, OUT, TS, Epi>(a, src, epi);
}

// ---------------------------------------------------------------- row pass
// Z[k] = (X[k] + conj X[M-k]) + i conj(W^k) (X[k] - conj X[M-k])   (C2R pre-processing)
template <typename C>
__device__ __forceinline__ C c2r_pre(C xa, C xb, C w) {
    C s = cadd(xa, cconj(xb)), d = csub(xa, cconj(xb));
    return cadd(s, cmul_i(cmulc(d, w)));
}
// X[k] = (Z[k] + conj Z[M-k]) - i W^k (Z[k] - conj Z[M-k])            (R2C post-processing)
template <typename C>
__device__ __forceinline__ C r2c_post(C za, C zb, C w) {
    C s = cadd(za, cconj(zb)), d = csub(za, cconj(zb));
    return csub(s, cmul_i(cmul(d, w)));
}

// Persistent double-buffered row pass: tiles of RB rows along dim 1
// (rows = (j, k) pairs), each row M+1 half-spectrum values, interleaved in
// shared memory as buf[n*TBP + b].
template <typename T, int IN, int OUT, bool MASK, typename TS, class Epi>
__device__ __forceinline__ void row_pass_kernel_body(PassArgs<T> a, const TS* __restrict__ src, Epi epi) {
    using C = cplx_t<T>;
    if (a.skip && *a.skip) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int M = a.g.m1;
    const int RB = a.rb, TBP = a.tbp;
    const size_t span = (size_t)(M + 1) * TBP;
    C* buf0 = reinterpret_cast<C*>(smem_raw);
    C* buf1 = buf0 + span;
    C* work = buf1 + span;
    __shared__ int s_rad[FFT_MAX_STAGES];
    load_radices(a.pl, s_rad);
    const C* tw = a.tw;
    if (a.tw_in_smem) {
        C* tws = work + span;
        for (int e = threadIdx.x; e < a.Ltab; e += blockDim.x) tws[e] = a.tw[e];
        tw = tws;
    }
    const int ntiles = (a.nrows + RB - 1) / RB;
    const C zero = mk((T)0, (T)0);
    const int half = M / 2;

    auto issue = [&](int t, C* dst) {
        const int r0 = t * RB, nr = min(RB, a.nrows - r0);
        if (IN == IN_REAL) {
            for (int e = threadIdx.x; e < M * RB; e += blockDim.x) {
                const int b = e / M, n = e % M;
                if (b < nr) cp_async<sizeof(C)>(&dst[n * TBP + b], a.real_in + (size_t)(r0 + b) * a.g.n1 + 2 * n);
                else dst[n * TBP + b] = zero;
            }
        } else {
            for (int e = threadIdx.x; e < (M + 1) * RB; e += blockDim.x) {
                const int b = e / (M + 1), n = e % (M + 1);
                if (b < nr) {
                    if (IN == IN_SPEC) cp_async<sizeof(C)>(&dst[n * TBP + b], a.spec + (size_t)(r0 + b) * a.g.ld1 + n);
                    else gather_issue<T>(decode1(a.g, n), src, &dst[n * TBP + b]);
                } else {
                    dst[n * TBP + b] = zero;
                }
            }
        }
    };

    Epi ep = epi;
    int t = blockIdx.x;
    if (t < ntiles) issue(t, buf0);
    cp_async_commit();
    for (int it = 0; t < ntiles; t += gridDim.x, ++it) {
        C* cur = (it & 1) ? buf1 : buf0;
        C* nxt = (it & 1) ? buf0 : buf1;
        if (t + (int)gridDim.x < ntiles) issue(t + gridDim.x, nxt);
        cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
        const int r0 = t * RB, nr = min(RB, a.nrows - r0);
        if (IN == IN_GATHER) {
            for (int n = threadIdx.x; n <= M; n += blockDim.x) cur[n * TBP] = gather_combine<T>(decode1(a.g, n), cur[n * TBP]);
            __syncthreads();
        }
        C* c1 = cur;
        if (IN != IN_REAL) {
            for (int e = threadIdx.x; e < (half + 1) * RB; e += blockDim.x) {
                const int b = e % RB, k = e / RB;
                if (k == 0) {
                    const C x0 = cur[b], xm = cur[M * TBP + b];
                    cur[b] = c2r_pre(x0, xm, tw[0]);
                } else if (2 * k == M) {
                    const C xk = cur[k * TBP + b];
                    cur[k * TBP + b] = c2r_pre(xk, xk, tw[k]);
                } else {
                    const C xk = cur[k * TBP + b], xm = cur[(M - k) * TBP + b];
                    cur[k * TBP + b] = c2r_pre(xk, xm, tw[k]);
                    cur[(M - k) * TBP + b] = c2r_pre(xm, xk, tw[M - k]);
                }
            }
            __syncthreads();
            c1 = fft_lines<T, true, true>(cur, work, s_rad, a.pl.nst, M, RB, TBP, tw, a.Ltab);
        }
        // scale and mask the real samples (x[2n], x[2n+1]) = (Re z[n], Im z[n])
        const T sc = (T)a.scale;
        for (int e = threadIdx.x; e < M * RB; e += blockDim.x) {
            const int b = e / M, n = e % M;
            if (b < nr) {
                C y = c1[n * TBP + b];
                y.x *= sc;
                y.y *= sc;
                if (MASK) {
                    const uint32_t w = a.maskw[(size_t)(r0 + b) * a.wpr + (n >> 4)];
                    const int sh = (2 * n) & 31;
                    if (!((w >> sh) & 1u)) y.x = (T)0;
                    if (!((w >> (sh + 1)) & 1u)) y.y = (T)0;
                }
                if (OUT == OUT_REAL) *reinterpret_cast<C*>(a.real_out + (size_t)(r0 + b) * a.g.n1 + 2 * n) = y;
                else c1[n * TBP + b] = y;
            }
        }
        if (OUT != OUT_REAL) {
            __syncthreads();
            C* other = (c1 == cur) ? work : cur;
            C* c2 = fft_lines<T, false, true>(c1, other, s_rad, a.pl.nst, M, RB, TBP, tw, a.Ltab);
            for (int e = threadIdx.x; e < (half + 1) * RB; e += blockDim.x) {
                const int b = e % RB, k = e / RB;
                if (k == 0) {
                    const C z0 = c2[b];
                    c2[b] = r2c_post(z0, z0, tw[0]);
                    c2[M * TBP + b] = mk((T)2 * (z0.x - z0.y), (T)0);
                } else if (2 * k == M) {
                    const C zk = c2[k * TBP + b];
                    c2[k * TBP + b] = r2c_post(zk, zk, tw[k]);
                } else {
                    const C zk = c2[k * TBP + b], zm = c2[(M - k) * TBP + b];
                    c2[k * TBP + b] = r2c_post(zk, zm, tw[k]);
                    c2[(M - k) * TBP + b] = r2c_post(zm, zk, tw[M - k]);
                }
            }
            __syncthreads();
            if (OUT == OUT_SPEC) {
                for (int e = threadIdx.x; e < (M + 1) * RB; e += blockDim.x) {
                    const int b = e / (M + 1), n = e % (M + 1);
                    if (b < nr) a.spec[(size_t)(r0 + b) * a.g.ld1 + n] = c2[n * TBP + b];
                }
            } else {   // 1D: one row, TBP == 1
                auto coord = [&](int e, int& i, int& j, int& k) -> bool { i = e; j = 0; k = 0; return true; };
                scatter_tile<T, SCATTER_UNROLL>(c2, M + 1, a.g, coord, ep);
            }
        }
        __syncthreads();
    }
    if (OUT == OUT_SCATTER) ep.finish();
}
template <typename T, int IN, int OUT, bool MASK, typename TS, class Epi>
__global__ void __launch_bounds__(256) row_pass_kernel(PassArgs<T> a, const TS* __restrict__ src, Epi epi) {
    row_pass_kernel_body<T, IN, OUT, MASK, TS, Epi>(a, src, epi);
}

// In-place row pass for rows too long to double-buffer (1D with large N):
// single tile, register-staged stages.
template <typename T, int IN, int OUT, bool MASK, typename TS, class Epi>
__global__ void __launch_bounds__(1024) row_pass_ip_kernel(PassArgs<T> a, const TS* __restrict__ src, Epi epi) {
    using C = cplx_t<T>;
    if (a.skip && *a.skip) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* buf = reinterpret_cast<C*>(smem_raw);
    const int M = a.g.m1;
    const int RB = a.rb, TBP = a.tbp;
    __shared__ int s_rad[FFT_MAX_STAGES];
    load_radices(a.pl, s_rad);
    constexpr bool PP = false;
    const size_t span = (size_t)(M + 1) * TBP;
    C* alt = nullptr;
    const C* tw = a.tw;
    if (a.tw_in_smem) {
        C* tws = buf + (PP ? 2 : 1) * span;
        for (int e = threadIdx.x; e < a.Ltab; e += blockDim.x) tws[e] = a.tw[e];
        tw = tws;
    }
    const int r0 = blockIdx.x * RB;
    const int nr = min(RB, a.nrows - r0);
    const C zero = mk((T)0, (T)0);

    // ---- load
    if (IN == IN_REAL) {
        for (int e = threadIdx.x; e < M * RB; e += blockDim.x) {
            const int b = e / M, n = e % M;
            C val = zero;
            if (b < nr) val = *reinterpret_cast<const C*>(a.real_in + (size_t)(r0 + b) * a.g.n1 + 2 * n);
            buf[n * TBP + b] = val;
        }
    } else {
        for (int e = threadIdx.x; e < (M + 1) * RB; e += blockDim.x) {
            const int b = e / (M + 1), n = e % (M + 1);
            C val = zero;
            if (b < nr) {
                if (IN == IN_SPEC) val = a.spec[(size_t)(r0 + b) * a.g.ld1 + n];
                else val = gather_val<T>(decode1(a.g, n), src);
            }
            buf[n * TBP + b] = val;
        }
    }
    __syncthreads();
    const int half = M / 2;
    C* cur = buf;
    if (IN != IN_REAL) {
        for (int e = threadIdx.x; e < (half + 1) * RB; e += blockDim.x) {
            const int b = e % RB, k = e / RB;
            if (k == 0) {
                const C x0 = buf[b], xm = buf[M * TBP + b];
                buf[b] = c2r_pre(x0, xm, tw[0]);
            } else if (2 * k == M) {
                const C xk = buf[k * TBP + b];
                buf[k * TBP + b] = c2r_pre(xk, xk, tw[k]);
            } else {
                const C xk = buf[k * TBP + b], xm = buf[(M - k) * TBP + b];
                buf[k * TBP + b] = c2r_pre(xk, xm, tw[k]);
                buf[(M - k) * TBP + b] = c2r_pre(xm, xk, tw[M - k]);
            }
        }
        __syncthreads();
        cur = fft_lines<T, true, PP>(buf, alt, s_rad, a.pl.nst, M, RB, TBP, tw, a.Ltab);
    }
    // ---- middle: scale and mask the real samples (x[2n], x[2n+1]) = (Re z[n], Im z[n])
    const T sc = (T)a.scale;
    for (int e = threadIdx.x; e < M * RB; e += blockDim.x) {
        const int b = e / M, n = e % M;
        if (b < nr) {
            C y = cur[n * TBP + b];
            y.x *= sc;
            y.y *= sc;
            if (MASK) {
                const uint32_t w = a.maskw[(size_t)(r0 + b) * a.wpr + (n >> 4)];
                const int sh = (2 * n) & 31;
                if (!((w >> sh) & 1u)) y.x = (T)0;
                if (!((w >> (sh + 1)) & 1u)) y.y = (T)0;
            }
            if (OUT == OUT_REAL) *reinterpret_cast<C*>(a.real_out + (size_t)(r0 + b) * a.g.n1 + 2 * n) = y;
            else cur[n * TBP + b] = y;
        }
    }
    if (OUT == OUT_REAL) return;
    __syncthreads();
    C* other = PP ? (cur == buf ? alt : buf) : nullptr;
    cur = fft_lines<T, false, PP>(cur, other, s_rad, a.pl.nst, M, RB, TBP, tw, a.Ltab);
    buf = cur;
    for (int e = threadIdx.x; e < (half + 1) * RB; e += blockDim.x) {
        const int b = e % RB, k = e / RB;
        if (k == 0) {
            const C z0 = buf[b];
            buf[b] = r2c_post(z0, z0, tw[0]);
            buf[M * TBP + b] = mk((T)2 * (z0.x - z0.y), (T)0);
        } else if (2 * k == M) {
            const C zk = buf[k * TBP + b];
            buf[k * TBP + b] = r2c_post(zk, zk, tw[k]);
        } else {
            const C zk = buf[k * TBP + b], zm = buf[(M - k) * TBP + b];
            buf[k * TBP + b] = r2c_post(zk, zm, tw[k]);
            buf[(M - k) * TBP + b] = r2c_post(zm, zk, tw[M - k]);
        }
    }
    __syncthreads();
    if (OUT == OUT_SPEC) {
        for (int e = threadIdx.x; e < (M + 1) * RB; e += blockDim.x) {
            const int b = e / (M + 1), n = e % (M + 1);
            if (b < nr) a.spec[(size_t)(r0 + b) * a.g.ld1 + n] = buf[n * TBP + b];
        }
    } else {
        Epi ep = epi;
        for (int n = threadIdx.x; n <= M; n += blockDim.x) scatter_one<T>(decode1(a.g, n), buf[n * TBP], ep);
        ep.finish();
    }
}

// ------------------------------------------------------------ host side
struct PassCfg {
    int tb = 0;          // lines per CTA (strided) / rows per CTA (row pass)
    int tbp = 0;         // padded line stride in shared memory
    int threads = 0;
    size_t smem = 0;
    int tw_in_smem = 0;
    int pp = 1;          // 1: persistent, double-buffered loads + ping-pong stages; 0: in place, one tile
    int tiles = 0;       // number of tiles of the pass
    dim3 grid;           // in-place path only; persistent grids are sized from occupancy at launch
};

// ------------------------------------------------------------ mask
// Observed-sample mask, one bit per real sample, rows of N1 bits padded to
// 32-bit words: every in-row bit set, padding clear; then the missing
// samples' bits cleared (duplicates are harmless).
static __global__ void mask_init_kernel(size_t words, int wpr, int n1, uint32_t* __restrict__ w) {
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < words; t += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(t % wpr);
        const int nb = min(32, n1 - 32 * c);
        w[t] = nb >= 32 ? 0xffffffffu : ((1u << nb) - 1u);
    }
}

static __global__ void mask_clear_kernel(const int64_t* __restrict__ idx, int64_t n, int n1, int wpr,
                                         uint32_t* __restrict__ w) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t v = idx[t];
        const int64_t r = v / n1;
        const int i = (int)(v - r * n1);
        atomicAnd(&w[r * wpr + (i >> 5)], ~(1u << (i & 31)));
    }
}

inline unsigned mask_blocks(long long n) { return (unsigned)std::max<long long>(1, std::min<long long>((n + 255) / 256, 4096)); }

// Long 1D rows (long1d.cuh): rows of M above L1D_MIN_M complex values run
// as M = P*Q over many CTAs.
constexpr int L1D_MIN_M = 2048;
constexpr int L1D_MAX_P = 4096;     // row length of the four-step row kernel
constexpr int L1D_MAX_Q = 768;      // line length of the first and last passes
constexpr int L1D_TB = 8;           // most lines per CTA of the first pass

// M = P*Q with Q the largest divisor of M not above sqrt(M) (nor L1D_MAX_Q),
// P = M/Q; false when P exceeds L1D_MAX_P
inline bool l1d_split(int M, int* P, int* Q) {
    int best = 0;
    for (int q = 2; (long long)q * q <= M && q <= L1D_MAX_Q; ++q)
        if (M % q == 0) best = q;
    if (!best || M / best > L1D_MAX_P) return false;
    *Q = best;
    *P = M / best;
    return true;
}

// W^e = exp(-2 pi i e / L), built on the device from the first octant with
// the exact symmetries of the roots of unity (sign changes and swaps only):
//   e in (L/2, L):    W^e = conj W^(L-e)                       (conjugation)
//   e in [L/4, L/2]:  W^e = -i W^(e-L/4)                       (quarter turn, 4 | L)
//   e in (L/8, L/4):  W^e = (-Im W^(L/4-e), -Re W^(L/4-e))     (reflection, 8 | L)
// What remains is computed directly as sincospi(2e/L) (2e/L is one rounding
// of an exact ratio; for 8 | L it lies in [0, 1/4]).  The table is symmetric
// bit for bit, as the real-input passes assume.
__device__ __forceinline__ double2 root_of_unity(long long e, long long L) {
    bool conj = false, rot = false, refl = false;
    if (2 * e > L) { e = L - e; conj = true; }
    if (L % 4 == 0 && 4 * e >= L) { e -= L / 4; rot = true; }
    if (L % 8 == 0 && 8 * e > L && 4 * e < L) { e = L / 4 - e; refl = true; }
    double sn, cs;
    sincospi((double)(2 * e) / (double)L, &sn, &cs);
    double re = cs, im = -sn;
    if (refl) { const double r2 = -im; im = -re; re = r2; }
    if (rot) { const double r2 = im; im = -re; re = r2; }
    if (conj) im = -im;
    return make_double2(re, im);
}

__device__ __forceinline__ void put_root(double2* o, double2 w) { *o = w; }
__device__ __forceinline__ void put_root(float2* o, double2 w) { *o = make_float2((float)w.x, (float)w.y); }

template <typename C>
__global__ void twiddle_kernel(int L, C* __restrict__ out) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < L; e += gridDim.x * blockDim.x)
        put_root(out + e, root_of_unity(e, L));
}

template <typename C>
inline cudaError_t launch_twiddles(int L, C* dst, cudaStream_t st) {
    const int blocks = std::max(1, std::min((L + 255) / 256, 1024));
    twiddle_kernel<C><<<blocks, 256, 0, st>>>(L, dst);
    return cudaGetLastError();
}

// Lines per CTA of the first pass (TB) and rows per CTA of the row pass (RB):
// as wide as shared memory allows (TB <= L1D_TB, RB <= 16) while each pass
// still launches about one CTA per SM (148 on B200; 128 for FP64, whose wide
// tiles measured faster down to that count).  A long row has only P and Q
// lines (a few hundred to a few thousand), so the widest tiles left most SMs
// idle (2^17: 32 CTAs per pass); the tile width changes no arithmetic.
inline void l1d_tiles(int P, int Q, size_t csize, int* TB, int* RB) {
    const int TARGET = csize >= 16 ? 128 : 148;
    int tb = L1D_TB;
    while (tb > 2 && (P + tb - 1) / tb < TARGET) tb /= 2;
    int rb = 1;
    while (rb < 16 && 2 * (size_t)P * (2 * rb) * csize <= 96 * 1024 && Q / (2 * rb) >= TARGET) rb *= 2;
    *TB = tb;
    *RB = rb;
}

template <typename T>
class FftOperator {
public:
    using C = cplx_t<T>;
    Geom g{};
    cudaStream_t stream = nullptr;
    C* spec = nullptr;              // (m1+1) x n2 x n3, pitch ld1
    uint32_t* maskw = nullptr;      // nullptr: no missing samples
    int wpr = 0;
    FftPlanDev plan1{}, plan2{}, plan3{};
    C* tw1 = nullptr;               // n1-th roots (row pass)
    C* tw2 = nullptr;
    C* tw3 = nullptr;
    PassCfg row_cfg, s2_cfg, s3_cfg;
    // two-level register passes (fft2.cuh): factor pairs, 0 when not used
    int s2_A = 0, s2_B = 0, s3_A = 0, s3_B = 0, r_A = 0, r_B = 0;
    size_t bytes = 0;
    bool owns = true;               // false: buffers belong to someone else; release() frees nothing
    const int4* pmap = nullptr;     // solver-order plane map (owned by the handle)
    // long 1D rows: M = l1P * l1Q (0 when the one-CTA row pass is used)
    int l1P = 0, l1Q = 0, l1RB = 0, l1TB = 0;
    FftPlanDev planP{}, planQ{};
    C* twP = nullptr;
    C* twQ = nullptr;
    PassCfg q_cfg;

    // stream-ordered allocations from this pool on `stream` when set (the
    // handle's), else plain cudaMalloc/cudaFree
    cudaMemPool_t pool = nullptr;

    ~FftOperator() { release(); }

    template <typename P>
    cudaError_t dalloc(P** p, size_t count) {
        void* q = nullptr;
        const cudaError_t e = pool ? cudaMallocFromPoolAsync(&q, sizeof(P) * count, pool, stream)
                                   : cudaMalloc(&q, sizeof(P) * count);
        *p = reinterpret_cast<P*>(q);
        return e;
    }
    void dfree(void* p) {
        if (!p) return;
        if (pool) cudaFreeAsync(p, stream);
        else cudaFree(p);
    }

    void release() {
        if (!owns) return;
        dfree(spec); spec = nullptr;
        dfree(maskw); maskw = nullptr;
        dfree(tw1); tw1 = nullptr;
        dfree(tw2); tw2 = nullptr;
        dfree(tw3); tw3 = nullptr;
        dfree(twP); twP = nullptr;
        dfree(twQ); twQ = nullptr;
    }

    // twiddle table of L entries, written on the device (stream-ordered: no
    // host computation, no copy)
    bool upload_table(int L, C** dst, std::string* err) {
        if (dalloc(dst, L) != cudaSuccess) { *err = "out of device memory (twiddles)"; return false; }
        if (launch_twiddles(L, *dst, stream) != cudaSuccess) { *err = "twiddle kernel launch failed"; return false; }
        return true;
    }

    // conservative dynamic shared-memory budget per CTA (B200 opt-in limit is 227 KB incl. static)
    static size_t smem_limit() { return 200 * 1024; }

    // Strided passes: three shared buffers of TB lines (two load stages + one
    // work buffer), TB a power of two chosen so a CTA takes ~64 KB.
    bool choose_strided(const FftPlanDev& pl, int Ltab, int n_lines, int n_outer, PassCfg* cfg, std::string* err) {
        const int L = pl.L;
        const size_t per_line = (size_t)L * sizeof(C);
        int tb = 16;
        while (tb > 2 && 3 * per_line * tb > 64 * 1024) tb /= 2;
        if (sizeof(T) == 8 && tb > 8) tb = 8;
        const size_t data = 3 * per_line * tb;
        if (data > smem_limit()) {
            *err = "transform length too large for the on-chip strided pass";
            return false;
        }
        cfg->tb = tb;
        cfg->tbp = tb;
        cfg->threads = 256;
        cfg->pp = 1;
        const size_t tws = (size_t)Ltab * sizeof(C);
        cfg->tw_in_smem = (data + tws <= smem_limit() && tws <= 32 * 1024) ? 1 : 0;
        cfg->smem = data + (cfg->tw_in_smem ? tws : 0);
        cfg->tiles = ((n_lines + tb - 1) / tb) * n_outer;
        cfg->grid = dim3(cfg->tiles, 1, 1);
        return true;
    }

    // Row passes: persistent with three buffers when they fit, else one
    // in-place tile per CTA (very long rows, 1D).
    bool choose_row(int nrows, PassCfg* cfg, std::string* err) {
        const int M = g.m1;
        const int Ltab = g.n1;
        const size_t tws = (size_t)Ltab * sizeof(C);
        int rb = 1;
        while (rb < 16 && rb * 2 <= nrows && 3 * (size_t)(M + 1) * (rb * 2 + 1) * sizeof(C) <= 72 * 1024) rb *= 2;
        const int tbp = rb > 1 ? rb + 1 : 1;
        const size_t one = (size_t)(M + 1) * tbp * sizeof(C);
        if (3 * one <= smem_limit()) {
            cfg->pp = 1;
            cfg->tb = rb;
            cfg->tbp = tbp;
            cfg->threads = 256;
            cfg->tw_in_smem = (3 * one + tws <= smem_limit() && tws <= 32 * 1024) ? 1 : 0;
            cfg->smem = 3 * one + (cfg->tw_in_smem ? tws : 0);
            cfg->tiles = (nrows + rb - 1) / rb;
            cfg->grid = dim3(cfg->tiles, 1, 1);
            return true;
        }
        // in place: the register-staged engine takes radices <= 8
        if (!make_fft_plan(M, &plan1, err, 8)) return false;
        for (rb = 1; rb >= 1; rb /= 2) {
            const int tp = 1;
            const size_t o1 = (size_t)(M + 1) * tp * sizeof(C);
            if (o1 > smem_limit()) break;
            int thr = ((M * rb + 7) / 8 + 31) / 32 * 32;
            thr = std::max(64, std::min(1024, thr));
            while (thr < 1024 && !plan_fits(plan1, rb, thr)) thr += 32;
            if (!plan_fits(plan1, rb, thr)) break;
            cfg->pp = 0;
            cfg->tb = rb;
            cfg->tbp = tp;
            cfg->threads = thr;
            cfg->tw_in_smem = (o1 + tws <= smem_limit() && tws <= 64 * 1024) ? 1 : 0;
            cfg->smem = o1 + (cfg->tw_in_smem ? tws : 0);
            cfg->tiles = (nrows + rb - 1) / rb;
            cfg->grid = dim3(cfg->tiles, 1, 1);
            return true;
        }
        *err = "dimension 1 too large for the on-chip row pass";
        return false;
    }

    // host_keep: N bytes (1 = observed) or nullptr for no mask
    // largest register radix of the double-buffered stages (FP64 keeps 20
    // complex values per thread, FP32 32)
    static int max_radix() { return 8; }

    // Use the two-level register passes where the line length factors into an
    // instantiated pair (FP64, 2D/3D).
    void choose_two_level();

    bool make_plans(std::string* err) {
        if (!make_fft_plan(g.m1, &plan1, err, max_radix())) return false;
        if (g.dim >= 2 && !make_fft_plan(g.n2, &plan2, err, max_radix())) return false;
        if (g.dim >= 3 && !make_fft_plan(g.n3, &plan3, err, max_radix())) return false;
        return true;
    }

    // dev_missing: n_missing 0-based linear indices of missing samples in
    // device memory (validated by the caller), or n_missing == 0 for no mask
    bool init(const Geom& geom, const int64_t* dev_missing, int64_t n_missing, cudaStream_t st, std::string* err) {
        g = geom;
        stream = st;
        const int nrows = g.n2 * g.n3;
        if (g.dim == 1 && g.m1 > L1D_MIN_M) {
            if (!l1d_split(g.m1, &l1P, &l1Q)) {
                *err = "1D length has no split M = P*Q with P <= 4096, Q <= 768";
                return false;
            }
            if (!make_fft_plan(l1P, &planP, err, max_radix()) || !make_fft_plan(l1Q, &planQ, err, max_radix()))
                return false;
            if (!choose_strided(planQ, l1Q, l1P, 1, &q_cfg, err)) return false;
            l1d_tiles(l1P, l1Q, sizeof(C), &l1TB, &l1RB);
            if (!upload_table(l1P, &twP, err) || !upload_table(l1Q, &twQ, err)) return false;
            plan1 = planP;   // unused by the long path; keeps the handle's plans defined
        } else {
            if (!make_plans(err)) return false;
            if (!choose_row(nrows, &row_cfg, err)) return false;
        }
        choose_two_level();
        if (g.dim >= 2 && !choose_strided(plan2, g.n2, g.m1 + 1, g.dim == 3 ? g.n3 : 1, &s2_cfg, err)) return false;
        if (g.dim >= 3 && !choose_strided(plan3, g.n3, g.m1 + 1, g.n2, &s3_cfg, err)) return false;
        if (!upload_table(g.n1, &tw1, err)) return false;
        if (g.dim >= 2 && !upload_table(g.n2, &tw2, err)) return false;
        if (g.dim >= 3 && !upload_table(g.n3, &tw3, err)) return false;
        const size_t spec_elems = (size_t)g.ld1 * g.n2 * g.n3;
        if (dalloc(&spec, spec_elems) != cudaSuccess) { *err = "out of device memory (spectrum)"; return false; }
        bytes += sizeof(C) * spec_elems;
        if (n_missing > 0) {
            wpr = (g.n1 + 31) / 32;
            const size_t words = (size_t)wpr * nrows;
            if (dalloc(&maskw, words) != cudaSuccess) { *err = "out of device memory (mask)"; return false; }
            bytes += sizeof(uint32_t) * words;
            mask_init_kernel<<<mask_blocks(words), 256, 0, stream>>>(words, wpr, g.n1, maskw);
            mask_clear_kernel<<<mask_blocks(n_missing), 256, 0, stream>>>(dev_missing, n_missing, g.n1, wpr, maskw);
            if (cudaGetLastError() != cudaSuccess) { *err = "mask construction failed"; return false; }
        }
        return true;
    }

    PassArgs<T> row_args(double scale, const T* real_in, T* real_out) const {
        PassArgs<T> a{};
        a.g = g; a.pl = plan1; a.tw = tw1; a.Ltab = g.n1; a.tw_in_smem = row_cfg.tw_in_smem;
        a.spec = spec; a.nrows = g.n2 * g.n3; a.rb = row_cfg.tb; a.tbp = row_cfg.tbp;
        a.maskw = maskw; a.wpr = wpr; a.scale = scale; a.real_in = real_in; a.real_out = real_out;
        return a;
    }
    // axis 2 or 3
    PassArgs<T> strided_args(int axis) const {
        PassArgs<T> a{};
        a.g = g;
        a.spec = spec;
        a.pmap = pmap;
        a.n_lines = g.m1 + 1;
        if (axis == 3) {
            a.pl = plan3; a.tw = tw3; a.Ltab = g.n3; a.tw_in_smem = s3_cfg.tw_in_smem;
            a.so = g.ld1; a.sx = (long long)g.ld1 * g.n2; a.jk_mode = 0; a.n_outer = g.n2;
        } else {
            a.pl = plan2; a.tw = tw2; a.Ltab = g.n2; a.tw_in_smem = s2_cfg.tw_in_smem;
            a.so = (long long)g.ld1 * g.n2; a.sx = g.ld1; a.jk_mode = g.dim == 3 ? 1 : 2; a.n_outer = g.dim == 3 ? g.n3 : 1;
        }
        return a;
    }
};

// Opts a kernel into the large dynamic shared-memory carve-out, once per
// (kernel, device).  The attribute is set under the lock and recorded only
// after it succeeded, so a thread that launches the kernel concurrently waits
// for it instead of launching before the opt-in (which fails the launch).
// The opt-in covers dynamic + static shared memory, so the dynamic limit set
// is the device's per-block opt-in maximum minus the kernel's static part.
// `always`: opt in even when the dynamic part alone is within 48 KB (a
// kernel whose static and dynamic shared memory together exceed it).
inline cudaError_t smem_optin_fn(const void* fn, size_t smem, bool always = false) {
    if (smem <= 48 * 1024 && !always) return cudaSuccess;
    int dev = 0;
    cudaGetDevice(&dev);
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, size_t> limit;   // dynamic bytes set
    std::lock_guard<std::mutex> lk(mu);
    auto it = limit.find({fn, dev});
    if (it != limit.end()) return smem <= it->second ? cudaSuccess : cudaErrorInvalidValue;
    int optin = 0;
    cudaError_t e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess) return e;
    cudaFuncAttributes fa{};
    e = cudaFuncGetAttributes(&fa, fn);
    if (e != cudaSuccess) return e;
    const int dyn = optin - (int)fa.sharedSizeBytes;
    if (dyn < 0 || (size_t)dyn < smem) return cudaErrorInvalidValue;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
    if (e == cudaSuccess) limit[{fn, dev}] = (size_t)dyn;
    return e;
}

template <typename K>
inline cudaError_t smem_optin(K kernel, size_t smem) {
    return smem_optin_fn((const void*)kernel, smem);
}

// Persistent grid: resident CTAs per SM (occupancy API, cached per kernel,
// device and configuration) times the SM count, capped by the tile count.
inline int persistent_grid(const void* fn, int threads, size_t smem, int tiles) {
    static std::mutex mu;
    static std::map<std::tuple<const void*, int, int, size_t>, int> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    const auto key = std::make_tuple(fn, dev, threads, smem);
    int per_sm = 0, sms = 0;
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = cache.find(key);
        if (it != cache.end()) per_sm = it->second;
    }
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (per_sm == 0) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem) != cudaSuccess || per_sm < 1) {
            cudaGetLastError();   // not left for the next launch check to report
            per_sm = 1;
        }
        std::lock_guard<std::mutex> lk(mu);
        cache[key] = per_sm;
    }
    const long long g = (long long)per_sm * (sms > 0 ? sms : 148);
    return (int)std::max<long long>(1, std::min<long long>(g, tiles));
}

// Launch helpers (template dispatch on TB).
template <typename T, bool INV, int IN, int OUT, typename TS, class Epi>
inline cudaError_t launch_strided(const PassCfg& c, const PassArgs<T>& a, const TS* src, const Epi& epi, cudaStream_t st) {
    cudaError_t e = cudaSuccess;
    switch (c.tb) {
#define CSIPM_TB_CASE(TBV)                                                                            \
        case TBV: {                                                                                   \
            auto k = strided_pass_kernel<T, TBV, INV, IN, OUT, TS, Epi>;                              \
            e = smem_optin(k, c.smem);                                                                \
            if (e != cudaSuccess) return e;                                                           \
            const int grid = persistent_grid((const void*)k, c.threads, c.smem, c.tiles);             \
            k<<<grid, c.threads, c.smem, st>>>(a, src, epi);                                          \
        } break;
        CSIPM_TB_CASE(2) CSIPM_TB_CASE(4) CSIPM_TB_CASE(8) CSIPM_TB_CASE(16)
#undef CSIPM_TB_CASE
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <typename T, int IN, int OUT, bool MASK, typename TS, class Epi>
inline cudaError_t launch_row(const PassCfg& c, const PassArgs<T>& a, const TS* src, const Epi& epi, cudaStream_t st) {
    if (c.pp) {
        auto k = row_pass_kernel<T, IN, OUT, MASK, TS, Epi>;
        cudaError_t e = smem_optin(k, c.smem);
        if (e != cudaSuccess) return e;
        const int grid = persistent_grid((const void*)k, c.threads, c.smem, c.tiles);
        k<<<grid, c.threads, c.smem, st>>>(a, src, epi);
    } else {
        auto k = row_pass_ip_kernel<T, IN, OUT, MASK, TS, Epi>;
        cudaError_t e = smem_optin(k, c.smem);
        if (e != cudaSuccess) return e;
        k<<<c.grid, c.threads, c.smem, st>>>(a, src, epi);
    }
    return cudaGetLastError();
}

}  // namespace csipm
