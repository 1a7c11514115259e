// Explicit instantiations of the two-level strided passes, FP32 (launchers in fft2_launch.cuh).
#include "fft2_launch.cuh"

namespace csipm {

#define CSIPM_INST_S2(T, INV, IN, OUT, TS, EPI) \
    template cudaError_t launch_strided2<T, INV, IN, OUT, TS, EPI>(int, int, const PassArgs<T>&, const TS*, const EPI&, cudaStream_t);
CSIPM_FFT2_STRIDED_LIST32(CSIPM_INST_S2)
#undef CSIPM_INST_S2

}  // namespace csipm
