// Launchers of the two-level register FFT passes (fft2.cuh): dispatch on the
// factor pair to the kernel instantiated for it.  The explicit
// instantiations are split over fft2_s64.cu, fft2_s32.cu, fft2_r64.cu and
// fft2_r32.cu so they compile in parallel.
#pragma once
#include "fft2.cuh"

namespace csipm {

template <typename T, bool INV, int IN, int OUT, typename TS, class Epi>
cudaError_t launch_strided2(int A, int B, const PassArgs<T>& a, const TS* src, const Epi& epi, cudaStream_t st) {
#define CSIPM_S2(AA, BB)                                                                                   \
    if (A == AA && B == BB) {                                                                              \
        constexpr int TB = fft2_tb<T, AA * BB>();                                                          \
        const dim3 grid((a.n_lines + TB - 1) / TB, a.n_outer, 1);                                          \
        strided2_kernel<T, AA, BB, INV, IN, OUT, TS, Epi><<<grid, TB * (AA > BB ? AA : BB), 0, st>>>(a, src, epi); \
        return cudaGetLastError();                                                                         \
    }
    CSIPM_FFT2_SPAIRS(CSIPM_S2)
#undef CSIPM_S2
    return cudaErrorInvalidValue;
}

// The bulk-staged persistent kernel for whole tiles of the spectrum-to-
// spectrum pass; false when the pass does not qualify (then the plain one).
template <typename T, int AA, int BB, bool MASK>
bool launch_row2b(const PassArgs<T>& a, cudaStream_t st, cudaError_t* err) {
    using Sh = Row2Shape<T, AA, BB>;
    const size_t tile_bytes = (size_t)Sh::ROWS * a.g.ld1 * sizeof(cplx_t<T>);
    if (a.nrows % Sh::ROWS || tile_bytes % 16 || ((uintptr_t)a.spec & 15) || a.g.ld1 < Sh::M + 1) return false;
    auto k = row2b_kernel<T, AA, BB, MASK>;
    const int threads = Sh::ROWS * Sh::NTL;
    const size_t dyn = tile_bytes + 2 * (size_t)Sh::M * sizeof(cplx_t<T>);   // tile + twiddle tables
    *err = smem_optin_fn((const void*)k, dyn, true);
    if (*err != cudaSuccess) return true;
    const int ntiles = a.nrows / Sh::ROWS;
    const int grid = persistent_grid((const void*)k, threads, dyn, ntiles);
    k<<<grid, threads, dyn, st>>>(a, ntiles);
    *err = cudaGetLastError();
    return true;
}

template <typename T, int IN, int OUT, bool MASK>
cudaError_t launch_row2(int A, int B, const PassArgs<T>& a, cudaStream_t st) {
#define CSIPM_R2(AA, BB)                                                                                   \
    if (A == AA && B == BB) {                                                                              \
        using Sh = Row2Shape<T, AA, BB>;                                                                   \
        if (IN == IN_SPEC && OUT == OUT_SPEC) {                                                            \
            cudaError_t e = cudaSuccess;                                                                   \
            if (launch_row2b<T, AA, BB, MASK>(a, st, &e)) return e;                                        \
        }                                                                                                  \
        const dim3 grid((a.nrows + Sh::ROWS - 1) / Sh::ROWS, 1, 1);                                        \
        row2_kernel<T, AA, BB, IN, OUT, MASK><<<grid, Sh::ROWS * Sh::NTL, 0, st>>>(a);                     \
        return cudaGetLastError();                                                                         \
    }
    CSIPM_FFT2_RPAIRS(CSIPM_R2)
#undef CSIPM_R2
    return cudaErrorInvalidValue;
}

}  // namespace csipm
