// Instantiations and launchers of the two-level register FFT passes
// (fft2.cuh) for the line lengths the library runs them on.
#include "fft2.cuh"

namespace csipm {

template <typename T, bool INV, int IN, int OUT, typename TS, class Epi>
cudaError_t launch_strided2(int A, int B, const PassArgs<T>& a, const TS* src, const Epi& epi, cudaStream_t st) {
    const dim3 grid((a.n_lines + FFT2_TB - 1) / FFT2_TB, a.n_outer, 1);
#define CSIPM_S2(AA, BB)                                                                                   \
    if (A == AA && B == BB) {                                                                              \
        strided2_kernel<T, AA, BB, INV, IN, OUT, TS, Epi><<<grid, FFT2_TB * (AA > BB ? AA : BB), 0, st>>>(a, src, epi); \
        return cudaGetLastError();                                                                         \
    }
    CSIPM_S2(16, 20) CSIPM_S2(16, 16) CSIPM_S2(10, 16) CSIPM_S2(8, 16) CSIPM_S2(8, 8)
#undef CSIPM_S2
    return cudaErrorInvalidValue;
}

template <typename T, int IN, int OUT, bool MASK>
cudaError_t launch_row2(int A, int B, const PassArgs<T>& a, cudaStream_t st) {
#define CSIPM_R2(AA, BB)                                                                                   \
    if (A == AA && B == BB) {                                                                              \
        using Sh = Row2Shape<T, AA, BB>;                                                                   \
        const dim3 grid((a.nrows + Sh::ROWS - 1) / Sh::ROWS, 1, 1);                                        \
        row2_kernel<T, AA, BB, IN, OUT, MASK><<<grid, Sh::ROWS * Sh::NTL, 0, st>>>(a);                     \
        return cudaGetLastError();                                                                         \
    }
    CSIPM_R2(10, 16) CSIPM_R2(8, 16) CSIPM_R2(8, 10) CSIPM_R2(8, 8) CSIPM_R2(16, 16)
#undef CSIPM_R2
    return cudaErrorInvalidValue;
}

#define CSIPM_INST_S2(INV, IN, OUT, EPI) \
    template cudaError_t launch_strided2<double, INV, IN, OUT, double, EPI>(int, int, const PassArgs<double>&, const double*, const EPI&, cudaStream_t);
CSIPM_INST_S2(true, IN_GATHER, OUT_SPEC, EpiStore<double>)
CSIPM_INST_S2(true, IN_SPEC, OUT_SPEC, EpiStore<double>)
CSIPM_INST_S2(false, IN_SPEC, OUT_SPEC, EpiStore<double>)
CSIPM_INST_S2(false, IN_SPEC, OUT_SCATTER, EpiStore<double>)
CSIPM_INST_S2(false, IN_SPEC, OUT_SCATTER, EpiCG<double>)
CSIPM_INST_S2(true, IN_SGATHER, OUT_SPEC, EpiStore<double>)
CSIPM_INST_S2(false, IN_SPEC, OUT_SSCATTER, EpiStore<double>)
CSIPM_INST_S2(false, IN_SPEC, OUT_SSCATTER, EpiCG<double>)
#undef CSIPM_INST_S2

template cudaError_t launch_row2<double, IN_SPEC, OUT_SPEC, true>(int, int, const PassArgs<double>&, cudaStream_t);
template cudaError_t launch_row2<double, IN_SPEC, OUT_SPEC, false>(int, int, const PassArgs<double>&, cudaStream_t);
template cudaError_t launch_row2<double, IN_SPEC, OUT_REAL, true>(int, int, const PassArgs<double>&, cudaStream_t);
template cudaError_t launch_row2<double, IN_SPEC, OUT_REAL, false>(int, int, const PassArgs<double>&, cudaStream_t);
template cudaError_t launch_row2<double, IN_REAL, OUT_SPEC, false>(int, int, const PassArgs<double>&, cudaStream_t);

}  // namespace csipm
