// Two-level register FFT passes: L = A*B.
//
// Step 1: each thread owns one residue t < B of a line and loads its A
// elements x[t + B*a] straight from global memory into registers (A loads in
// flight per thread), runs DFT_A, multiplies by W_L^{t*ka} and writes the A
// results to shared memory.  Step 2: thread s < A reads its B values, runs
// DFT_B and owns the outputs X[s + A*kb].  One shared-memory round trip per
// transform (the Stockham engine needs one per radix stage).
//
// In the row pass the inverse transform (A, B) leaves thread s with
// z[s + A*kb]; the forward transform is run with the factors swapped (B, A),
// whose first step wants exactly those elements, so C2R -> mask -> R2C costs
// two exchanges plus one for the R2C post-processing.
#pragma once
#include <cuda_runtime.h>

#include "bulk.cuh"
#include "fft_device.cuh"
#include "operator.cuh"

namespace csipm {

// Lines per CTA of the strided two-level pass of length L: 128 B per access
// (8 FP64 or 16 FP32 complex) while the CTA's lines fit the 48 KB of static
// shared memory, else the most that fit (lines above 384 points: 4 or 2).
template <typename T, int L> constexpr int fft2_tb() {
    constexpr int full = sizeof(T) == 8 ? 8 : 16;
    constexpr int fit = (47 * 1024) / (L * 2 * (int)sizeof(T));   // 1 KB left for the reductions' arrays
    return fit >= full ? full : (fit >= 8 ? 8 : (fit >= 4 ? 4 : 2));
}
// fewest lines per CTA of any strided two-level pass (sizes the grid-reduction
// workspace of the scatter passes, whose grids have (N1/2+1)/TB columns)
constexpr int FFT2_TB_MIN = 2;

// twiddle of the strided pass: W_L^e (forward) from a table of L-th roots
template <bool INV, typename C>
__device__ __forceinline__ C tw_apply(C v, const C* __restrict__ tw, int e) {
    if (e == 0) return v;
    const C w = tw[e];
    return INV ? cmulc(v, w) : cmul(v, w);
}

// ------------------------------------------------------------ strided pass
// CTAs per SM the register allocation of a strided pass must allow, by
// precision, CTA size (NT threads) and pass kind, as measured on B200 at
// 256^3 and 320^3: more CTAs hide the gather/scatter load latency (the
// scatter epilogue would otherwise take 88 FP32 / 148 FP64 registers and
// leave 2 CTAs per SM), while the plain FP64 pass of 160-thread CTAs runs
// fastest unconstrained.  (An explicit 1 lets the compiler use up to 255
// registers, more than it picks with no bound at all.)
template <typename T, int IN, int OUT, int NT> constexpr int fft2_min_ctas() {
    constexpr bool scatter = OUT == OUT_SSCATTER || OUT == OUT_SCATTER;
    if (sizeof(T) == 4) return scatter ? 3 : (NT <= 256 ? 4 : 3);
    if (NT <= 128) return 4;
    return scatter ? 3 : ((IN == IN_SGATHER || IN == IN_GATHER) ? 4 : 1);
}

template <typename T, int A, int B, bool INV, int IN, int OUT, typename TS, class Epi>
__global__ void __launch_bounds__(fft2_tb<T, A * B>() * (A > B ? A : B),
                                  (fft2_min_ctas<T, IN, OUT, fft2_tb<T, A * B>() * (A > B ? A : B)>()))
strided2_kernel(PassArgs<T> a, const TS* __restrict__ src, Epi epi) {
    using C = cplx_t<T>;
    constexpr int L = A * B;
    constexpr int TB = fft2_tb<T, L>();
    if (a.skip && *a.skip) return;
    __shared__ C S[L * TB];
    const int b = threadIdx.x % TB, t = threadIdx.x / TB;
    const int i0 = blockIdx.x * TB, o = blockIdx.y;
    const int nb = min(TB, a.n_lines - i0);
    const bool live = b < nb;
    const long long base = i0 + b + (long long)o * a.so;
    const C* __restrict__ tw = a.tw;    // L-th roots (Ltab == L)
    const C zero = mk((T)0, (T)0);
    // each thread keeps one dim-1 position for the whole tile: interior
    // positions (all but i = 0 and i = M1) take the short decode
    const int ii = i0 + b;
    const bool interior = ii >= 1 && ii <= a.g.m1 - 1;

    // Solver-order scatter: the epilogue operands of this thread's first
    // SC_U outputs are requested now, so their latency hides behind step 1,
    // the exchange and DFT_B (later chunks are prefetched one chunk ahead).
    // FP32 only: in FP64 the extra live registers cost more occupancy than
    // the early loads win.
    constexpr int SC_U = 4;
    constexpr bool SC_EARLY = sizeof(T) == 4;
    typename Epi::Pre2 sc_pre[SC_U];
    int64_t sc_p0 = 0, sc_ps = 0;
    const bool sc_own = OUT == OUT_SSCATTER && t < A && live && interior;
    if constexpr (OUT == OUT_SSCATTER) {
        if (sc_own) {
            int j0, k0s;
            jk_of(a.jk_mode, o, t, j0, k0s);
            sc_p0 = sol_pair(a.g, ii, j0, k0s);
            sc_ps = (a.jk_mode == 0 ? (int64_t)a.g.n2 : (int64_t)1) * (a.g.m1 - 1) * A;
            if constexpr (SC_EARLY) {
#pragma unroll
                for (int q = 0; q < SC_U; ++q)
                    if (q < B) sc_pre[q] = epi.pre2(sc_p0 + q * sc_ps);
            }
        }
    }
    // ---- step 1: thread t < B owns x = t + B*a
    if (t < B) {
        C v[A];
        if constexpr (IN == IN_SGATHER) {
            // interior lines: one base pair index plus q times a fixed stride
            // (the branch is per thread and outside the element loop, so the
            // A loads issue back to back)
            if (live && interior) {
                const cplx_t<TS>* __restrict__ s2 = reinterpret_cast<const cplx_t<TS>*>(src);
                int j0, k0;
                jk_of(a.jk_mode, o, t, j0, k0);
                const int64_t p0 = sol_pair(a.g, ii, j0, k0);
                const int64_t ps = (a.jk_mode == 0 ? (int64_t)a.g.n2 : (int64_t)1) * (a.g.m1 - 1) * B;
                const T r = (T)0.7071067811865476;
#pragma unroll
                for (int q = 0; q < A; ++q) {
                    const cplx_t<TS> w = s2[p0 + q * ps];
                    v[q] = mk((T)w.x * r, (T)w.y * r);
                }
            } else {
#pragma unroll
                for (int q = 0; q < A; ++q) {
                    const int x = t + B * q;
                    int j, k;
                    jk_of(a.jk_mode, o, x, j, k);
                    if (live) {
                        const int4 t4 = a.pmap[((ii == 0 ? 0 : 1) * a.g.n3 + k) * a.g.n2 + j];
                        v[q] = gather_val<T>(MapEntry{t4.x, t4.y, t4.z, t4.w}, src);
                    } else {
                        v[q] = zero;
                    }
                }
            }
        } else {
#pragma unroll
        for (int q = 0; q < A; ++q) {
            const int x = t + B * q;
            if (!live) {
                v[q] = zero;
            } else if constexpr (IN == IN_SPEC) {
                v[q] = a.spec[base + (long long)x * a.sx];
            } else if constexpr (IN == IN_SGATHER) {
                int j, k;
                jk_of(a.jk_mode, o, x, j, k);
                if (interior) {
                    const cplx_t<TS> w = reinterpret_cast<const cplx_t<TS>*>(src)[sol_pair(a.g, ii, j, k)];
                    const T r = (T)0.7071067811865476;
                    v[q] = mk((T)w.x * r, (T)w.y * r);
                } else {   // planes i = 0, M1: tabulated entries (no per-element decode)
                    const int4 t4 = a.pmap[((ii == 0 ? 0 : 1) * a.g.n3 + k) * a.g.n2 + j];
                    v[q] = gather_val<T>(MapEntry{t4.x, t4.y, t4.z, t4.w}, src);
                }
            } else {
                int j, k;
                jk_of(a.jk_mode, o, x, j, k);
                const MapEntry en = interior ? decode_interior(a.g, ii, j, k) : decode(a.g, ii, j, k);
                v[q] = gather_val<T>(en, src);
            }
        }
        }
        Dft<A, INV, T>::run(v);
#pragma unroll
        for (int ka = 0; ka < A; ++ka) S[(ka * B + t) * TB + b] = tw_apply<INV>(v[ka], tw, t * ka);
    }
    __syncthreads();
    // ---- step 2: thread s < A owns X[s + A*kb]
    Epi ep = epi;
    if (t < A && live) {
        const int s = t;
        C u[B];
#pragma unroll
        for (int q = 0; q < B; ++q) u[q] = S[(s * B + q) * TB + b];
        Dft<B, INV, T>::run(u);
        if constexpr (OUT == OUT_SPEC) {
#pragma unroll
            for (int kb = 0; kb < B; ++kb) a.spec[base + (long long)(s + A * kb) * a.sx] = u[kb];
        } else if (OUT == OUT_SSCATTER && interior) {
            // pair index of x = s + A*kb: one base plus kb times a fixed stride
            // (sc_p0, sc_ps); FP32 loads the operands one chunk ahead of their use
            if constexpr (SC_EARLY) {
#pragma unroll
                for (int k0 = 0; k0 < B; k0 += SC_U) {
                    typename Epi::Pre2 nxt[SC_U];
                    if (k0 + SC_U < B) {
#pragma unroll
                        for (int q = 0; q < SC_U; ++q)
                            if (k0 + SC_U + q < B) nxt[q] = ep.pre2(sc_p0 + (k0 + SC_U + q) * sc_ps);
                    }
#pragma unroll
                    for (int q = 0; q < SC_U; ++q)
                        if (k0 + q < B)
                            ep.put2(sc_p0 + (k0 + q) * sc_ps, (T)SQRT2_D * u[k0 + q].x, (T)SQRT2_D * u[k0 + q].y,
                                    sc_pre[q]);
                    if (k0 + SC_U < B) {
#pragma unroll
                        for (int q = 0; q < SC_U; ++q) sc_pre[q] = nxt[q];
                    }
                }
            } else {
#pragma unroll
                for (int k0 = 0; k0 < B; k0 += SC_U) {
#pragma unroll
                    for (int q = 0; q < SC_U; ++q)
                        if (k0 + q < B) sc_pre[q] = ep.pre2(sc_p0 + (k0 + q) * sc_ps);
#pragma unroll
                    for (int q = 0; q < SC_U; ++q)
                        if (k0 + q < B)
                            ep.put2(sc_p0 + (k0 + q) * sc_ps, (T)SQRT2_D * u[k0 + q].x, (T)SQRT2_D * u[k0 + q].y,
                                    sc_pre[q]);
                }
            }
        } else {
            constexpr int U = 2;
#pragma unroll
            for (int k0 = 0; k0 < B; k0 += U) {
                MapEntry en[U];
                typename Epi::Pre pr[U], pi[U];
#pragma unroll
                for (int q = 0; q < U; ++q) {
                    if (k0 + q < B) {
                        int j, k;
                        jk_of(a.jk_mode, o, s + A * (k0 + q), j, k);
                        if (OUT == OUT_SSCATTER) {   // planes i = 0, M1 in solver order: tabulated
                            const int4 t4 = a.pmap[((ii == 0 ? 0 : 1) * a.g.n3 + k) * a.g.n2 + j];
                            en[q] = MapEntry{t4.x, t4.y, t4.z, t4.w};
                        } else {
                            en[q] = interior ? decode_interior(a.g, ii, j, k) : decode(a.g, ii, j, k);
                        }
                        if (en[q].src) {
                            pr[q] = ep.pre(en[q].re);
                            if (en[q].kind != KIND_VERT) pi[q] = ep.pre(en[q].im);
                        }
                    }
                }
#pragma unroll
                for (int q = 0; q < U; ++q) {
                    if (k0 + q < B && en[q].src) {
                        const C v = u[k0 + q];
                        if (en[q].kind == KIND_VERT) {
                            ep.put(en[q].re, (double)v.x, pr[q]);
                        } else {
                            ep.put(en[q].re, SQRT2_D * (double)v.x, pr[q]);
                            ep.put(en[q].im, (en[q].kind == KIND_PLUS ? SQRT2_D : -SQRT2_D) * (double)v.y, pi[q]);
                        }
                    }
                }
            }
        }
    }
    if (OUT == OUT_SCATTER || OUT == OUT_SSCATTER) ep.finish();
}

// ---------------------------------------------------------------- row pass
// Rows per CTA of the row pass: as many as fit in 48 KB of static shared
// memory, at most 8 (16-row CTAs of 256 threads measured 12% slower at
// M = 160 on B200, though they fill whole warps in both mappings).
constexpr int row2_rows(int per_row_bytes) {
    const int r0 = (48 * 1024) / per_row_bytes;
    return r0 > 8 ? 8 : (r0 < 1 ? 1 : r0);
}

// M = A*B half-spectrum length (dim-1 complex FFT length); rows of M+1 values.
template <typename T, int A, int B> struct Row2Shape {
    static constexpr int M = A * B;
    static constexpr int X1 = A * (B + 1);          // inverse exchange  [ka][t],  t-stride 1, ka-stride B+1
    static constexpr int X2 = B * (A + 1);          // forward exchange  [kb][s],  s-stride 1, kb-stride A+1
    static constexpr int XC = X1 > X2 ? X1 : X2;
    static constexpr int BASE = XC + M + 1;         // exchange area + natural-order spectrum for R2C post
    // row pitch = A (mod 16) complex: in the A-task phases a half-warp spans
    // two rows, and the next row's lanes then land on the banks after the
    // first row's (8-byte complex: 16 bank pairs; 16-byte: 8 bank quads)
    static constexpr int PER_ROW = BASE + (((A - BASE) % 16) + 16) % 16;
    static constexpr int NTL = A > B ? A : B;
    static constexpr int ROWS = row2_rows(PER_ROW * (int)sizeof(cplx_t<T>));
    // Minimum resident CTAs per SM in the launch bound.  FP32: 1, which lets
    // ptxas give the (10, 16) pass 102 registers (5 CTAs per SM) where the
    // bound without a CTA count gave 72 (7 CTAs per SM): 0.129 -> 0.115 ms
    // at 320^3 on B200.  FP64 with A < 16: as many as shared memory holds
    // (228 KB per SM, 1 KB reserved per CTA) at up to 128 registers per
    // thread: the (10, 16) pass keeps 4 CTAs per SM with 128 registers
    // (104 with no CTA count); same-box A/B at 320^3: FP64 solve
    // 0.0763 -> 0.0747 s, mixed 0.0529 -> 0.0524 s, where a 96-register cap
    // (5 CTAs per SM) measured no gain and a count of 1 took 164 registers
    // (3 CTAs per SM).  A 64-register cap on the FP32 passes, and any cap on
    // (16, 16), spilled.
    static constexpr int SMEM = ROWS * PER_ROW * (int)sizeof(cplx_t<T>);
    static constexpr int BY_SMEM = (228 * 1024) / (SMEM + 1024);
    static constexpr int BY_REGS = 65536 / (ROWS * NTL * 128);
    static constexpr int MINB_RAW = BY_SMEM < BY_REGS ? BY_SMEM : BY_REGS;
    static constexpr int MINB = (sizeof(T) != 8 || A == 16 || MINB_RAW < 1) ? 1 : MINB_RAW;
    // Bulk-staged variant (row2b_kernel): one tile buffer of ROWS rows of
    // M+1 values and two M-entry twiddle tables beside the exchange area;
    // resident CTAs per SM: as many as
    // shared memory holds at up to ~100 (FP32) / ~168 (FP64) registers per
    // thread, at most 6.
    static constexpr int TILE = (ROWS * (M + 1) + 2 * M) * (int)sizeof(cplx_t<T>);
    static constexpr int BY_SMEM_B = (228 * 1024) / (SMEM + TILE + 1024);
    static constexpr int BY_REGS_B = 65536 / (ROWS * NTL * (sizeof(T) == 8 ? 168 : 100));
    static constexpr int MINB_B0 = BY_SMEM_B < BY_REGS_B ? BY_SMEM_B : BY_REGS_B;
    static constexpr int MINB_B = MINB_B0 < 1 ? 1 : (MINB_B0 > 6 ? 6 : MINB_B0);
};

// Two thread mappings share the CTA: the B-task phases (inverse step 1,
// forward step 2, C2R/R2C pre/post-processing) give each row NTL = B
// consecutive threads; the A-task phases (inverse step 2, scale + mask,
// forward step 1: the B-point DFTs) give each row A consecutive threads, so
// ROWS*A threads work in whole warps instead of A of every B lanes.
template <typename T, int A, int B, int IN, int OUT, bool MASK>
__global__ void __launch_bounds__(Row2Shape<T, A, B>::ROWS * Row2Shape<T, A, B>::NTL, Row2Shape<T, A, B>::MINB)
row2_kernel(PassArgs<T> a) {
    using C = cplx_t<T>;
    using Sh = Row2Shape<T, A, B>;
    constexpr int M = Sh::M;
    constexpr int NTL = Sh::NTL;
    static_assert(A <= B, "row pass factors are ordered A <= B");
    if (a.skip && *a.skip) return;
    __shared__ C S[Sh::ROWS * Sh::PER_ROW];
    // B-task mapping
    const int r = threadIdx.x / NTL, t = threadIdx.x % NTL;
    const int row = blockIdx.x * Sh::ROWS + r;
    const bool live = row < a.nrows;
    C* X = S + r * Sh::PER_ROW;           // exchange area of this row
    C* P = X + Sh::XC;                    // natural-order spectrum (R2C post)
    // A-task mapping
    const bool ta = threadIdx.x < Sh::ROWS * A;
    const int ra = threadIdx.x / A, s = threadIdx.x % A;
    const int rowa = blockIdx.x * Sh::ROWS + ra;
    const bool livea = ta && rowa < a.nrows;
    C* XA = S + (ta ? ra : 0) * Sh::PER_ROW;
    const C* __restrict__ tw = a.tw;      // N1-th roots, W_M^e = tw[2e]
    const C zero = mk((T)0, (T)0);
    const T sc = (T)a.scale;

    // z[s + A*kb] of the A-task s after the inverse transform (or the load)
    C z[B];
    if (IN == IN_REAL) {
        if (ta) {
#pragma unroll
            for (int kb = 0; kb < B; ++kb) {
                const int n = s + A * kb;
                z[kb] = livea ? *reinterpret_cast<const C*>(a.real_in + (size_t)rowa * a.g.n1 + 2 * n) : zero;
            }
        }
    } else {
        // ---- inverse step 1 (B-task t): C2R pre-processing at load
        {
            C v[A];
            const C* rowp = a.spec + (size_t)row * a.g.ld1;
#pragma unroll
            for (int q = 0; q < A; ++q) {
                const int x = t + B * q;
                if (live) {
                    const C xa = rowp[x], xb = rowp[M - x];
                    v[q] = c2r_pre(xa, xb, tw[x]);
                } else {
                    v[q] = zero;
                }
            }
            Dft<A, true, T>::run(v);
#pragma unroll
            for (int ka = 0; ka < A; ++ka) {
                C w = v[ka];
                const int e = t * ka;
                if (e) w = cmulc(w, tw[2 * e]);
                X[ka * (B + 1) + t] = w;
            }
        }
        __syncthreads();
        // ---- inverse step 2 (A-task s)
        if (ta) {
#pragma unroll
            for (int q = 0; q < B; ++q) z[q] = XA[s * (B + 1) + q];
            Dft<B, true, T>::run(z);
        }
        __syncthreads();   // the exchange area is reused by the forward transform
    }
    // ---- scale and mask the real samples (x[2n], x[2n+1]) = z[n], n = s + A*kb
    if (ta) {
#pragma unroll
        for (int kb = 0; kb < B; ++kb) {
            const int n = s + A * kb;
            C y = z[kb];
            y.x *= sc;
            y.y *= sc;
            if (MASK && livea) {
                const uint32_t w = a.maskw[(size_t)rowa * a.wpr + (n >> 4)];
                const int sh = (2 * n) & 31;
                if (!((w >> sh) & 1u)) y.x = (T)0;
                if (!((w >> (sh + 1)) & 1u)) y.y = (T)0;
            }
            z[kb] = y;
            if (OUT == OUT_REAL && livea) *reinterpret_cast<C*>(a.real_out + (size_t)rowa * a.g.n1 + 2 * n) = y;
        }
    }
    if (OUT == OUT_REAL) return;
    // ---- forward transform with factors (B, A): step 1 (A-task s) on its own z
    if (ta) {
        Dft<B, false, T>::run(z);
#pragma unroll
        for (int kb = 0; kb < B; ++kb) {
            C w = z[kb];
            const int e = s * kb;
            if (e) w = cmul(w, tw[2 * e]);
            XA[kb * (A + 1) + s] = w;
        }
    }
    __syncthreads();
    // step 2 (B-task t): outputs Z[t + B*ka]
    {
        C u[A];
#pragma unroll
        for (int q = 0; q < A; ++q) u[q] = X[t * (A + 1) + q];
        Dft<A, false, T>::run(u);
#pragma unroll
        for (int ka = 0; ka < A; ++ka) P[t + B * ka] = u[ka];
    }
    __syncthreads();
    // ---- R2C post-processing and coalesced store of the M+1 values
    if (live) {
        C* rowp = a.spec + (size_t)row * a.g.ld1;
        for (int k = t; k <= M; k += NTL) {
            if (k == 0 || k == M) {
                const C z0 = P[0];
                rowp[k] = k == 0 ? r2c_post(z0, z0, tw[0]) : mk((T)2 * (z0.x - z0.y), (T)0);
            } else {
                rowp[k] = r2c_post(P[k], P[M - k], tw[k]);
            }
        }
    }
}

// ---------------------------------------------------------------- row pass, bulk-staged
// The spectrum-to-spectrum row pass (C2R, scale + mask, R2C) as a persistent
// kernel whose input rows arrive by bulk asynchronous copies (cp.async.bulk,
// completed on an mbarrier).  A tile is ROWS consecutive rows, which are
// contiguous in the half spectrum (pitch ld1), so one copy brings a tile.
// Once the first step of the inverse transform has read the tile into
// registers, the buffer is free and thread 0 issues the copy of the CTA's
// next tile; it lands while the rest of this tile is transformed, so the
// loads of a tile no longer stall the SM at its start (the plain kernel's
// long-scoreboard stalls).  Results go out with ordinary coalesced stores.
// The host uses it for whole tiles only (nrows a multiple of ROWS, tile bytes
// a multiple of 16, 16-byte aligned spectrum).
//
// Every wait is bounded: if a tile's copy has not completed after
// ROW2B_WAIT_LIMIT polls, the CTA writes NaN into that tile's rows (so the
// solve reports a non-finite iterate), counts the event in
// g_row2b_timeouts and returns.
constexpr int ROW2B_WAIT_LIMIT = 1 << 22;
static __device__ int g_row2b_timeouts;

template <typename T, int A, int B, bool MASK>
__global__ void __launch_bounds__(Row2Shape<T, A, B>::ROWS * Row2Shape<T, A, B>::NTL, Row2Shape<T, A, B>::MINB_B)
row2b_kernel(PassArgs<T> a, int ntiles) {
    using C = cplx_t<T>;
    using Sh = Row2Shape<T, A, B>;
    constexpr int M = Sh::M;
    constexpr int NTL = Sh::NTL;
    constexpr int R = Sh::ROWS;
    static_assert(A <= B, "row pass factors are ordered A <= B");
    if (a.skip && *a.skip) return;
    __shared__ C S[R * Sh::PER_ROW];
    // the twiddles of the two inner steps, laid out for their readers: the
    // inverse step 1 reads W^(t*ka) with consecutive t across lanes, the
    // forward step 1 W^(s*kb) with consecutive s; read from the N1-th root
    // table those are strided (a line per lane), which made the L1 pipe the
    // pass's bound
    __shared__ __align__(8) uint64_t full;
    __shared__ int s_ok;
    // dynamic: the tile buffer (R rows at pitch ld1), then T1 and T2
    extern __shared__ __align__(16) unsigned char row2b_dyn[];
    C* buf = reinterpret_cast<C*>(row2b_dyn);
    const int ld = a.g.ld1;
    const size_t tile_elems = (size_t)R * ld;
    C* T1 = buf + tile_elems;   // T1[ka*B + t] = W_M^(t*ka)
    C* T2 = T1 + M;             // T2[kb*A + s] = W_M^(s*kb)
    const uint32_t tile_bytes = (uint32_t)(tile_elems * sizeof(C));
    // B-task mapping
    const int r = threadIdx.x / NTL, t = threadIdx.x % NTL;
    C* X = S + r * Sh::PER_ROW;
    C* P = X + Sh::XC;
    const C* rowp = buf + (size_t)r * ld;
    // A-task mapping
    const bool ta = threadIdx.x < R * A;
    const int ra = threadIdx.x / A, s = threadIdx.x % A;
    C* XA = S + (ta ? ra : 0) * Sh::PER_ROW;
    const C* __restrict__ tw = a.tw;
    const T sc = (T)a.scale;
    const uint32_t bar = smem_u32(&full);
    const uint32_t dst = smem_u32(buf);

    for (int e = threadIdx.x; e < M; e += blockDim.x) {
        const int ka = e / B, tt = e % B;
        T1[e] = tw[2 * ((tt * ka) % M)];
        const int kb = e / A, ss = e % A;
        T2[e] = tw[2 * ((ss * kb) % M)];
    }
    int tile = blockIdx.x;
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        mbar_fence_init();
        if (tile < ntiles) {
            mbar_arrive_expect_tx(bar, tile_bytes);
            bulk_g2s(dst, a.spec + (size_t)tile * tile_elems, tile_bytes, bar);
        }
    }
    __syncthreads();
    uint32_t parity = 0;
    for (; tile < ntiles; tile += gridDim.x, parity ^= 1u) {
        // thread 0 waits (bounded) and tells the others; then every thread
        // observes the completed phase itself, which returns at once
        if (threadIdx.x == 0) s_ok = mbar_wait_bounded(bar, parity, ROW2B_WAIT_LIMIT) ? 1 : 0;
        __syncthreads();
        if (!s_ok) {
            if (threadIdx.x == 0) atomicAdd(&g_row2b_timeouts, 1);
            const T nan = (T)__int_as_float(0x7fc00000);
            C* out = a.spec + (size_t)tile * tile_elems;
            for (size_t e = threadIdx.x; e < tile_elems; e += blockDim.x) out[e] = mk(nan, nan);
            return;
        }
        mbar_try_wait(bar, parity);
        const int row = tile * R + r;
        // ---- inverse step 1 (B-task t): C2R pre-processing from the tile
        {
            C v[A];
#pragma unroll
            for (int q = 0; q < A; ++q) {
                const int x = t + B * q;
                v[q] = c2r_pre(rowp[x], rowp[M - x], tw[x]);
            }
            Dft<A, true, T>::run(v);
#pragma unroll
            for (int ka = 0; ka < A; ++ka) {
                C w = v[ka];
                if (t * ka) w = cmulc(w, T1[ka * B + t]);
                X[ka * (B + 1) + t] = w;
            }
        }
        __syncthreads();
        // the tile buffer is free: bring the next tile while this one is transformed
        if (threadIdx.x == 0) {
            const int next = tile + gridDim.x;
            if (next < ntiles) {
                fence_proxy_async_smem();
                mbar_arrive_expect_tx(bar, tile_bytes);
                bulk_g2s(dst, a.spec + (size_t)next * tile_elems, tile_bytes, bar);
            }
        }
        // ---- inverse step 2 (A-task s)
        C z[B];
        if (ta) {
#pragma unroll
            for (int q = 0; q < B; ++q) z[q] = XA[s * (B + 1) + q];
            Dft<B, true, T>::run(z);
        }
        __syncthreads();   // the exchange area is reused by the forward transform
        // ---- scale and mask the real samples (x[2n], x[2n+1]) = z[n], n = s + A*kb
        const int rowa = tile * R + ra;
        if (ta) {
#pragma unroll
            for (int kb = 0; kb < B; ++kb) {
                const int n = s + A * kb;
                C y = z[kb];
                y.x *= sc;
                y.y *= sc;
                if (MASK) {
                    const uint32_t w = a.maskw[(size_t)rowa * a.wpr + (n >> 4)];
                    const int sh = (2 * n) & 31;
                    if (!((w >> sh) & 1u)) y.x = (T)0;
                    if (!((w >> (sh + 1)) & 1u)) y.y = (T)0;
                }
                z[kb] = y;
            }
            // ---- forward transform with factors (B, A): step 1 (A-task s)
            Dft<B, false, T>::run(z);
#pragma unroll
            for (int kb = 0; kb < B; ++kb) {
                C w = z[kb];
                if (s * kb) w = cmul(w, T2[kb * A + s]);
                XA[kb * (A + 1) + s] = w;
            }
        }
        __syncthreads();
        // step 2 (B-task t): outputs Z[t + B*ka]
        {
            C u[A];
#pragma unroll
            for (int q = 0; q < A; ++q) u[q] = X[t * (A + 1) + q];
            Dft<A, false, T>::run(u);
#pragma unroll
            for (int ka = 0; ka < A; ++ka) P[t + B * ka] = u[ka];
        }
        __syncthreads();
        // ---- R2C post-processing and coalesced store of the M+1 values
        {
            C* rowg = a.spec + (size_t)row * ld;
            for (int k = t; k <= M; k += NTL) {
                if (k == 0 || k == M) {
                    const C z0 = P[0];
                    rowg[k] = k == 0 ? r2c_post(z0, z0, tw[0]) : mk((T)2 * (z0.x - z0.y), (T)0);
                } else {
                    rowg[k] = r2c_post(P[k], P[M - k], tw[k]);
                }
            }
        }
        __syncthreads();   // P and the exchange area are reused by the next tile
    }
}

// --------------------------------------------------------------- dispatch
// Factor L = A*B for the two-level passes (A, B among the register DFT sizes, A <= B, balanced);
// returns false when L has no supported factorisation.
inline bool fft2_factor(int L, int* A, int* B) {
    static const int sup[] = {32, 30, 27, 25, 24, 20, 18, 16, 15, 12, 10, 9, 8, 6, 5, 4};
    int bestA = 0, bestB = 0;
    for (int b : sup) {
        if (L % b) continue;
        const int a = L / b;
        bool ok = false;
        for (int s : sup) ok |= (s == a);
        if (!ok || a > b) continue;
        if (!bestA || a > bestA) { bestA = a; bestB = b; }
    }
    if (!bestA) return false;
    *A = bestA;
    *B = bestB;
    return true;
}

// The (A, B) pairs the library instantiates (fft2_*.cu): the lengths of the
// 320^3 / 256^3 / 2D 1024^2 workloads (strided 1024 = 32 x 32 at 2 FP64 or
// 4 FP32 lines per CTA) and the common dimension lengths of the serving
// stream's recoveries (3D sides of 32-128, 2D sides of 128-1024, factors
// 2, 3, 5), picked from its length histogram weighted by work (pairs whose
// kernels spill registers heavily, or that the autotuner found slower than
// Stockham, are left to Stockham).
#define CSIPM_FFT2_SPAIRS(X) \
    X(16, 20) X(16, 16) X(10, 16) X(8, 16) X(8, 8) X(10, 12) X(9, 12) X(8, 10) X(8, 9) X(9, 10) X(10, 10) \
    X(8, 12) X(5, 8) X(6, 8) X(6, 9) X(6, 6) X(6, 10) X(5, 10) X(4, 8) X(32, 32) X(20, 20) X(25, 32) \
    X(15, 16) X(15, 20) X(12, 15) X(20, 25) X(27, 32) X(18, 24) X(30, 32) X(24, 24) X(30, 30) X(24, 25) \
    X(18, 18) X(18, 20) X(27, 30)
#define CSIPM_FFT2_RPAIRS(X) \
    X(10, 16) X(8, 16) X(8, 10) X(8, 8) X(16, 16) X(16, 32) X(6, 10) X(6, 6) X(6, 9) X(5, 10) X(4, 8) \
    X(5, 9) X(5, 8) X(4, 6) X(6, 8) X(4, 5) X(5, 6) X(5, 5) X(12, 15) X(15, 15) X(4, 4) X(15, 20) \
    X(18, 20) X(18, 25) X(18, 18) X(9, 18) X(20, 24) X(15, 18) X(12, 18) X(16, 18) X(10, 20) X(16, 20)
inline bool fft2_strided_pair(int A, int B) {
#define CSIPM_IS_PAIR(AA, BB) if (A == AA && B == BB) return true;
    CSIPM_FFT2_SPAIRS(CSIPM_IS_PAIR)
    return false;
}
inline bool fft2_row_pair(int A, int B) {
    CSIPM_FFT2_RPAIRS(CSIPM_IS_PAIR)
#undef CSIPM_IS_PAIR
    return false;
}

template <typename T, bool INV, int IN, int OUT, typename TS, class Epi>
cudaError_t launch_strided2(int A, int B, const PassArgs<T>& a, const TS* src, const Epi& epi, cudaStream_t st);

template <typename T, int IN, int OUT, bool MASK>
cudaError_t launch_row2(int A, int B, const PassArgs<T>& a, cudaStream_t st);

// The instantiations of the two-level passes (fft2.cu): (T, INV, IN, OUT, TS,
// Epi) and (T, IN, OUT, MASK).  Fft2S / Fft2R tell the dispatch which exist.
#define CSIPM_FFT2_STRIDED_LIST64(X)                                 \
    X(double, true, IN_GATHER, OUT_SPEC, double, EpiStore<double>)   \
    X(double, true, IN_SPEC, OUT_SPEC, double, EpiStore<double>)     \
    X(double, false, IN_SPEC, OUT_SPEC, double, EpiStore<double>)    \
    X(double, false, IN_SPEC, OUT_SCATTER, double, EpiStore<double>) \
    X(double, false, IN_SPEC, OUT_SCATTER, double, EpiCG<double>)    \
    X(double, true, IN_SGATHER, OUT_SPEC, double, EpiStore<double>)  \
    X(double, false, IN_SPEC, OUT_SSCATTER, double, EpiStore<double>) \
    X(double, false, IN_SPEC, OUT_SSCATTER, double, EpiCG<double>)
#define CSIPM_FFT2_STRIDED_LIST32(X)                                 \
    X(float, true, IN_GATHER, OUT_SPEC, float, EpiStore<double>)     \
    X(float, true, IN_SGATHER, OUT_SPEC, float, EpiStore<double>)    \
    X(float, true, IN_SPEC, OUT_SPEC, double, EpiStore<double>)      \
    X(float, false, IN_SPEC, OUT_SPEC, double, EpiStore<double>)     \
    X(float, false, IN_SPEC, OUT_SCATTER, double, EpiCG<float>)      \
    X(float, false, IN_SPEC, OUT_SSCATTER, double, EpiCG<float>)
#define CSIPM_FFT2_STRIDED_LIST(X) CSIPM_FFT2_STRIDED_LIST64(X) CSIPM_FFT2_STRIDED_LIST32(X)

#define CSIPM_FFT2_ROW_LIST64(X)         \
    X(double, IN_SPEC, OUT_SPEC, true)   \
    X(double, IN_SPEC, OUT_SPEC, false)  \
    X(double, IN_SPEC, OUT_REAL, true)   \
    X(double, IN_SPEC, OUT_REAL, false)  \
    X(double, IN_REAL, OUT_SPEC, false)
#define CSIPM_FFT2_ROW_LIST32(X)         \
    X(float, IN_SPEC, OUT_SPEC, true)    \
    X(float, IN_SPEC, OUT_SPEC, false)
#define CSIPM_FFT2_ROW_LIST(X) CSIPM_FFT2_ROW_LIST64(X) CSIPM_FFT2_ROW_LIST32(X)

template <typename T, bool INV, int IN, int OUT, typename TS, class Epi>
struct Fft2S { static constexpr bool value = false; };
template <typename T, int IN, int OUT, bool MASK>
struct Fft2R { static constexpr bool value = false; };
#define CSIPM_FFT2_HAS_S(T, INV, IN, OUT, TS, EPI) \
    template <> struct Fft2S<T, INV, IN, OUT, TS, EPI> { static constexpr bool value = true; };
#define CSIPM_FFT2_HAS_R(T, IN, OUT, MASK) \
    template <> struct Fft2R<T, IN, OUT, MASK> { static constexpr bool value = true; };
CSIPM_FFT2_STRIDED_LIST(CSIPM_FFT2_HAS_S)
CSIPM_FFT2_ROW_LIST(CSIPM_FFT2_HAS_R)
#undef CSIPM_FFT2_HAS_S
#undef CSIPM_FFT2_HAS_R

}  // namespace csipm

namespace csipm {

template <typename T>
inline void FftOperator<T>::choose_two_level() {
    s2_A = s2_B = s3_A = s3_B = r_A = r_B = 0;
    if (g.dim < 2) return;
    int A = 0, B = 0;
    if (fft2_factor(g.n2, &A, &B) && fft2_strided_pair(A, B)) { s2_A = A; s2_B = B; }
    if (g.dim == 3 && fft2_factor(g.n3, &A, &B) && fft2_strided_pair(A, B)) { s3_A = A; s3_B = B; }
    if (fft2_factor(g.m1, &A, &B) && fft2_row_pair(A, B)) { r_A = A; r_B = B; }
}

}  // namespace csipm
