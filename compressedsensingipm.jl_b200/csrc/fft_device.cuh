// Mixed-radix Stockham FFT over lines held in shared memory.
//
// A CTA holds TB interleaved lines of length L in shared memory, element
// (x, b) at buf[x*TBP + b] (b fastest, TBP >= TB).  Two stage engines:
//   ping-pong (default): each stage reads one buffer and writes the other, one
//     butterfly per loop trip, so only R complex values are live per thread;
//   in place (lines too long to double-buffer): each thread loads all its
//     butterflies into registers, the block synchronises, then it stores;
//     this path may spill registers and is only used for very long rows.
// Stage s with radix
// R and Ns = product of the radices before it maps butterfly u of line b to
//   inputs  x = u + r*(L/R)                       (r = 0..R-1)
//   outputs x = (u - u%Ns)*R + u%Ns + r*Ns
// with twiddle W_{Ns*R}^{(u%Ns)*r} on input r, giving natural order after the
// last stage.  Twiddles come from a table of Ltab-th roots of unity
// W^e = exp(-2*pi*i*e/Ltab) (Ltab a multiple of L); the inverse transform uses
// their conjugates.  Radices 2, 3, 4, 5, 7, 8 have register butterflies; any
// other prime is done as a direct DFT.
#pragma once
#include "cplx.cuh"
#include "roots.h"

namespace csipm {

constexpr int FFT_MAX_STAGES = 24;

struct FftPlanDev {
    int L;                       // transform length
    int nst;                     // number of stages
    int rad[FFT_MAX_STAGES];     // radices, in order
};

// per-thread register budget: about 8 complex values per stage
template <int R> struct MaxItems { static constexpr int v = (8 + R - 1) / R; };
constexpr int GENERIC_MAX_ITEMS = 8;

// ---------------------------------------------------------------- butterflies
template <bool INV, typename C> __device__ __forceinline__ C rot_mi(C a) {   // a * (-i) forward, a * (+i) inverse
    return INV ? cmul_i(a) : cmul_mi(a);
}

template <int R, bool INV, typename T> struct Dft;

template <bool INV, typename T> struct Dft<2, INV, T> {
    using C = cplx_t<T>;
    __device__ __forceinline__ static void run(C* a) {
        C t = a[0];
        a[0] = cadd(t, a[1]);
        a[1] = csub(t, a[1]);
    }
};

template <bool INV, typename T> struct Dft<4, INV, T> {
    using C = cplx_t<T>;
    __device__ __forceinline__ static void run(C* a) {
        C t0 = cadd(a[0], a[2]), t1 = csub(a[0], a[2]);
        C t2 = cadd(a[1], a[3]), t3 = rot_mi<INV>(csub(a[1], a[3]));
        a[0] = cadd(t0, t2);
        a[2] = csub(t0, t2);
        a[1] = cadd(t1, t3);
        a[3] = csub(t1, t3);
    }
};

template <bool INV, typename T> struct Dft<8, INV, T> {
    using C = cplx_t<T>;
    __device__ __forceinline__ static void run(C* a) {
        const T h = (T)0.7071067811865476;   // sqrt(2)/2
        C e[4] = {a[0], a[2], a[4], a[6]};
        C o[4] = {a[1], a[3], a[5], a[7]};
        Dft<4, INV, T>::run(e);
        Dft<4, INV, T>::run(o);
        // o[k] *= W8^k  (W8 = exp(-i*pi/4) forward)
        C o1, o2, o3;
        if (!INV) {
            o1 = mk((o[1].x + o[1].y) * h, (o[1].y - o[1].x) * h);
            o2 = cmul_mi(o[2]);
            o3 = mk((o[3].y - o[3].x) * h, -(o[3].x + o[3].y) * h);
        } else {
            o1 = mk((o[1].x - o[1].y) * h, (o[1].x + o[1].y) * h);
            o2 = cmul_i(o[2]);
            o3 = mk(-(o[3].x + o[3].y) * h, (o[3].x - o[3].y) * h);
        }
        a[0] = cadd(e[0], o[0]); a[4] = csub(e[0], o[0]);
        a[1] = cadd(e[1], o1);   a[5] = csub(e[1], o1);
        a[2] = cadd(e[2], o2);   a[6] = csub(e[2], o2);
        a[3] = cadd(e[3], o3);   a[7] = csub(e[3], o3);
    }
};

template <bool INV, typename T> struct Dft<3, INV, T> {
    using C = cplx_t<T>;
    __device__ __forceinline__ static void run(C* a) {
        const T s = (T)0.8660254037844386;   // sin(2*pi/3)
        C t1 = cadd(a[1], a[2]), t2 = csub(a[1], a[2]);
        C m = mk(a[0].x - (T)0.5 * t1.x, a[0].y - (T)0.5 * t1.y);
        a[0] = cadd(a[0], t1);
        // forward: y1 = m - i*s*t2, y2 = m + i*s*t2
        C st = mk(s * t2.x, s * t2.y);
        C ist = cmul_i(st);
        if (!INV) { a[1] = csub(m, ist); a[2] = cadd(m, ist); }
        else      { a[1] = cadd(m, ist); a[2] = csub(m, ist); }
    }
};

template <bool INV, typename T> struct Dft<5, INV, T> {
    using C = cplx_t<T>;
    __device__ __forceinline__ static void run(C* a) {
        const T c1 = (T)0.30901699437494745, c2 = (T)-0.8090169943749475;
        const T s1 = (T)0.9510565162951535, s2 = (T)0.5877852522924731;
        C t1 = cadd(a[1], a[4]), t2 = cadd(a[2], a[3]);
        C t3 = csub(a[1], a[4]), t4 = csub(a[2], a[3]);
        C b1 = mk(a[0].x + c1 * t1.x + c2 * t2.x, a[0].y + c1 * t1.y + c2 * t2.y);
        C b2 = mk(a[0].x + c2 * t1.x + c1 * t2.x, a[0].y + c2 * t1.y + c1 * t2.y);
        C e1 = mk(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y);
        C e2 = mk(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y);
        a[0] = cadd(a[0], cadd(t1, t2));
        C ie1 = cmul_i(e1), ie2 = cmul_i(e2);
        if (!INV) { a[1] = csub(b1, ie1); a[4] = cadd(b1, ie1); a[2] = csub(b2, ie2); a[3] = cadd(b2, ie2); }
        else      { a[1] = cadd(b1, ie1); a[4] = csub(b1, ie1); a[2] = cadd(b2, ie2); a[3] = csub(b2, ie2); }
    }
};

template <bool INV, typename T> struct Dft<7, INV, T> {
    using C = cplx_t<T>;
    __device__ __forceinline__ static void run(C* a) {
        const T c1 = (T)0.6234898018587335, c2 = (T)-0.2225209339563144, c3 = (T)-0.9009688679024191;
        const T s1 = (T)0.7818314824680298, s2 = (T)0.9749279121818236, s3 = (T)0.4338837391175581;
        C t1 = cadd(a[1], a[6]), t2 = cadd(a[2], a[5]), t3 = cadd(a[3], a[4]);
        C d1 = csub(a[1], a[6]), d2 = csub(a[2], a[5]), d3 = csub(a[3], a[4]);
        C x0 = a[0];
        C b1 = mk(x0.x + c1 * t1.x + c2 * t2.x + c3 * t3.x, x0.y + c1 * t1.y + c2 * t2.y + c3 * t3.y);
        C b2 = mk(x0.x + c2 * t1.x + c3 * t2.x + c1 * t3.x, x0.y + c2 * t1.y + c3 * t2.y + c1 * t3.y);
        C b3 = mk(x0.x + c3 * t1.x + c1 * t2.x + c2 * t3.x, x0.y + c3 * t1.y + c1 * t2.y + c2 * t3.y);
        C e1 = mk(s1 * d1.x + s2 * d2.x + s3 * d3.x, s1 * d1.y + s2 * d2.y + s3 * d3.y);
        C e2 = mk(s2 * d1.x - s3 * d2.x - s1 * d3.x, s2 * d1.y - s3 * d2.y - s1 * d3.y);
        C e3 = mk(s3 * d1.x - s1 * d2.x + s2 * d3.x, s3 * d1.y - s1 * d2.y + s2 * d3.y);
        a[0] = cadd(x0, cadd(t1, cadd(t2, t3)));
        C i1 = cmul_i(e1), i2 = cmul_i(e2), i3 = cmul_i(e3);
        if (!INV) {
            a[1] = csub(b1, i1); a[6] = cadd(b1, i1);
            a[2] = csub(b2, i2); a[5] = cadd(b2, i2);
            a[3] = csub(b3, i3); a[4] = cadd(b3, i3);
        } else {
            a[1] = cadd(b1, i1); a[6] = csub(b1, i1);
            a[2] = cadd(b2, i2); a[5] = csub(b2, i2);
            a[3] = cadd(b3, i3); a[4] = csub(b3, i3);
        }
    }
};

// Composite radix R = R1*R2 in registers: R2 DFTs of size R1 over
// a[n2 + R2*n1], twiddles W_R^{n2*k1} (compile-time constants), then R1 DFTs
// of size R2; output X[k1 + R1*k2].
template <int R1, int R2, bool INV, typename T> struct DftComp {
    using C = cplx_t<T>;
    static constexpr int R = R1 * R2;
    __device__ __forceinline__ static void run(C* a) {
        C y[R];
#pragma unroll
        for (int n2 = 0; n2 < R2; ++n2) {
            C t[R1];
#pragma unroll
            for (int n1 = 0; n1 < R1; ++n1) t[n1] = a[n2 + R2 * n1];
            Dft<R1, INV, T>::run(t);
#pragma unroll
            for (int k1 = 0; k1 < R1; ++k1) {
                const int m = (n2 * k1) % R;
                C v = t[k1];
                if (m != 0) {
                    const C w = mk((T)RootTab<R>::re(m), (T)RootTab<R>::im(m));
                    v = INV ? cmulc(v, w) : cmul(v, w);
                }
                y[k1 * R2 + n2] = v;
            }
        }
#pragma unroll
        for (int k1 = 0; k1 < R1; ++k1) {
            C t[R2];
#pragma unroll
            for (int n2 = 0; n2 < R2; ++n2) t[n2] = y[k1 * R2 + n2];
            Dft<R2, INV, T>::run(t);
#pragma unroll
            for (int k2 = 0; k2 < R2; ++k2) a[k1 + R1 * k2] = t[k2];
        }
    }
};

template <bool INV, typename T> struct Dft<6, INV, T> : DftComp<2, 3, INV, T> {};
template <bool INV, typename T> struct Dft<9, INV, T> : DftComp<3, 3, INV, T> {};
template <bool INV, typename T> struct Dft<10, INV, T> : DftComp<2, 5, INV, T> {};
template <bool INV, typename T> struct Dft<12, INV, T> : DftComp<4, 3, INV, T> {};
template <bool INV, typename T> struct Dft<15, INV, T> : DftComp<3, 5, INV, T> {};
template <bool INV, typename T> struct Dft<16, INV, T> : DftComp<4, 4, INV, T> {};
template <bool INV, typename T> struct Dft<20, INV, T> : DftComp<4, 5, INV, T> {};
template <bool INV, typename T> struct Dft<25, INV, T> : DftComp<5, 5, INV, T> {};
template <bool INV, typename T> struct Dft<32, INV, T> : DftComp<8, 4, INV, T> {};
template <bool INV, typename T> struct Dft<18, INV, T> : DftComp<2, 9, INV, T> {};
template <bool INV, typename T> struct Dft<24, INV, T> : DftComp<8, 3, INV, T> {};
template <bool INV, typename T> struct Dft<27, INV, T> : DftComp<3, 9, INV, T> {};
template <bool INV, typename T> struct Dft<30, INV, T> : DftComp<5, 6, INV, T> {};

// ------------------------------------------------------------------- stages
template <typename T, int R, bool INV>
__device__ __forceinline__ void stage_pp(const cplx_t<T>* __restrict__ in, cplx_t<T>* __restrict__ out, int L, int TB,
                                         int TBP, int Ns, const cplx_t<T>* __restrict__ tw, int step) {
    using C = cplx_t<T>;
    const int m = L / R;
    const int nitems = TB * m;
    for (int w = threadIdx.x; w < nitems; w += blockDim.x) {
        const int b = w % TB, u = w / TB, k = u % Ns;
        C v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = in[(u + r * m) * TBP + b];
        if (Ns > 1) {
#pragma unroll
            for (int r = 1; r < R; ++r) v[r] = twmul<INV>(v[r], tw[k * r * step]);
        }
        Dft<R, INV, T>::run(v);
        const int o = ((u - k) * R + k) * TBP + b;
#pragma unroll
        for (int r = 0; r < R; ++r) out[o + r * Ns * TBP] = v[r];
    }
}

// direct DFT of an arbitrary (prime) radix p: one output per loop trip
template <typename T, bool INV>
__device__ __forceinline__ void stage_generic_pp(const cplx_t<T>* __restrict__ in, cplx_t<T>* __restrict__ out, int L,
                                                 int TB, int TBP, int Ns, int p, const cplx_t<T>* __restrict__ tw,
                                                 int step, int Ltab) {
    using C = cplx_t<T>;
    const int m = L / p;
    const int nitems = TB * L;   // (b, u, r_out)
    for (int w = threadIdx.x; w < nitems; w += blockDim.x) {
        const int b = w % TB, rest = w / TB;
        const int u = rest % m, ro = rest / m, k = u % Ns;
        // exponent of input t: t*step*(k + ro*Ns)  (mod Ltab)
        const int e0 = (int)(((long long)step * (k + ro * Ns)) % Ltab);
        C acc = mk((T)0, (T)0);
        int e = 0;
        for (int t = 0; t < p; ++t) {
            acc = cadd(acc, twmul<INV>(in[(u + t * m) * TBP + b], tw[e]));
            e += e0;
            if (e >= Ltab) e -= Ltab;
        }
        out[((u - k) * p + k + ro * Ns) * TBP + b] = acc;
    }
}

template <typename T, int R, bool INV>
__device__ __forceinline__ void stage_ip(cplx_t<T>* __restrict__ buf, int L, int TB, int TBP, int Ns,
                                      const cplx_t<T>* __restrict__ tw, int step) {
    using C = cplx_t<T>;
    constexpr int MI = MaxItems<R>::v;
    const int m = L / R;
    const int nitems = TB * m;
    const int tid = threadIdx.x, nthr = blockDim.x;
    C v[MI][R];
    int oidx[MI];
#pragma unroll
    for (int it = 0; it < MI; ++it) {
        const int w = tid + it * nthr;
        oidx[it] = -1;
        if (w < nitems) {
            const int b = w % TB, u = w / TB, k = u % Ns;
#pragma unroll
            for (int r = 0; r < R; ++r) v[it][r] = buf[(u + r * m) * TBP + b];
            if (Ns > 1) {
#pragma unroll
                for (int r = 1; r < R; ++r) v[it][r] = twmul<INV>(v[it][r], tw[k * r * step]);
            }
            Dft<R, INV, T>::run(v[it]);
            oidx[it] = ((u - k) * R + k) * TBP + b;
        }
    }
    __syncthreads();
#pragma unroll
    for (int it = 0; it < MI; ++it) {
        if (oidx[it] >= 0) {
#pragma unroll
            for (int r = 0; r < R; ++r) buf[oidx[it] + r * Ns * TBP] = v[it][r];
        }
    }
    __syncthreads();
}

template <typename T, bool INV>
__device__ __forceinline__ void stage_generic_ip(cplx_t<T>* __restrict__ buf, int L, int TB, int TBP, int Ns, int p,
                                              const cplx_t<T>* __restrict__ tw, int step, int Ltab) {
    using C = cplx_t<T>;
    const int m = L / p;
    const int nitems = TB * L;
    const int tid = threadIdx.x, nthr = blockDim.x;
    C res[GENERIC_MAX_ITEMS];
    int oidx[GENERIC_MAX_ITEMS];
#pragma unroll
    for (int it = 0; it < GENERIC_MAX_ITEMS; ++it) {
        const int w = tid + it * nthr;
        oidx[it] = -1;
        if (w < nitems) {
            const int b = w % TB, rest = w / TB;
            const int u = rest % m, ro = rest / m, k = u % Ns;
            const int e0 = (int)(((long long)step * (k + ro * Ns)) % Ltab);
            C acc = mk((T)0, (T)0);
            int e = 0;
            for (int t = 0; t < p; ++t) {
                acc = cadd(acc, twmul<INV>(buf[(u + t * m) * TBP + b], tw[e]));
                e += e0;
                if (e >= Ltab) e -= Ltab;
            }
            res[it] = acc;
            oidx[it] = ((u - k) * p + k + ro * Ns) * TBP + b;
        }
    }
    __syncthreads();
#pragma unroll
    for (int it = 0; it < GENERIC_MAX_ITEMS; ++it)
        if (oidx[it] >= 0) buf[oidx[it]] = res[it];
    __syncthreads();
}

// Copy a plan's radix list into shared memory with compile-time indices, so the
// kernel-parameter struct is never indexed dynamically (which would force a
// local-memory copy of the whole parameter block).  Followed by a barrier in
// the caller before first use.
__device__ __forceinline__ void load_radices(const FftPlanDev& pl, int* s_rad) {
#pragma unroll
    for (int s = 0; s < FFT_MAX_STAGES; ++s)
        if (threadIdx.x == s) s_rad[s] = pl.rad[s];
}

// Full transform of TB interleaved lines of length L.  PP: data starts in
// `buf`, `alt` is the second buffer; returns the buffer holding the result.
// In place (PP == false): `alt` is unused and `buf` is returned.
// Every thread of the block must call this (it contains barriers).
template <typename T, bool INV, bool PP>
__device__ cplx_t<T>* fft_lines(cplx_t<T>* buf, cplx_t<T>* alt, const int* s_rad, int nst, int L, int TB, int TBP,
                                const cplx_t<T>* __restrict__ tw, int Ltab) {
    int Ns = 1;
    cplx_t<T>* in = buf;
    cplx_t<T>* out = alt;
#pragma unroll 1
    for (int s = 0; s < nst; ++s) {
        const int R = s_rad[s];
        const int step = Ltab / (Ns * R);
        if (PP) {
            switch (R) {
                case 2: stage_pp<T, 2, INV>(in, out, L, TB, TBP, Ns, tw, step); break;
                case 3: stage_pp<T, 3, INV>(in, out, L, TB, TBP, Ns, tw, step); break;
                case 4: stage_pp<T, 4, INV>(in, out, L, TB, TBP, Ns, tw, step); break;
                case 5: stage_pp<T, 5, INV>(in, out, L, TB, TBP, Ns, tw, step); break;
                case 6: stage_pp<T, 6, INV>(in, out, L, TB, TBP, Ns, tw, step); break;
                case 7: stage_pp<T, 7, INV>(in, out, L, TB, TBP, Ns, tw, step); break;
                case 8: stage_pp<T, 8, INV>(in, out, L, TB, TBP, Ns, tw, step); break;
                case 9: stage_pp<T, 9, INV>(in, out, L, TB, TBP, Ns, tw, step); break;
                case 10: stage_pp<T, 10, INV>(in, out, L, TB, TBP, Ns, tw, step); break;
                case 12: stage_pp<T, 12, INV>(in, out, L, TB, TBP, Ns, tw, step); break;
                case 15: stage_pp<T, 15, INV>(in, out, L, TB, TBP, Ns, tw, step); break;
                case 16: stage_pp<T, 16, INV>(in, out, L, TB, TBP, Ns, tw, step); break;
                case 20: stage_pp<T, 20, INV>(in, out, L, TB, TBP, Ns, tw, step); break;
                case 25: stage_pp<T, 25, INV>(in, out, L, TB, TBP, Ns, tw, step); break;
                case 32: stage_pp<T, 32, INV>(in, out, L, TB, TBP, Ns, tw, step); break;
                default: stage_generic_pp<T, INV>(in, out, L, TB, TBP, Ns, R, tw, step, Ltab); break;
            }
            __syncthreads();
            cplx_t<T>* t = in; in = out; out = t;
        } else {
            switch (R) {
                case 2: stage_ip<T, 2, INV>(buf, L, TB, TBP, Ns, tw, step); break;
                case 3: stage_ip<T, 3, INV>(buf, L, TB, TBP, Ns, tw, step); break;
                case 4: stage_ip<T, 4, INV>(buf, L, TB, TBP, Ns, tw, step); break;
                case 5: stage_ip<T, 5, INV>(buf, L, TB, TBP, Ns, tw, step); break;
                case 7: stage_ip<T, 7, INV>(buf, L, TB, TBP, Ns, tw, step); break;
                case 8: stage_ip<T, 8, INV>(buf, L, TB, TBP, Ns, tw, step); break;
                default: stage_generic_ip<T, INV>(buf, L, TB, TBP, Ns, R, tw, step, Ltab); break;
            }
        }
        Ns *= R;
    }
    return PP ? in : buf;
}

}  // namespace csipm
