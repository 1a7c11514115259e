// Explicit instantiations of the two-level row passes, FP32 (launchers in fft2_launch.cuh).
#include "fft2_launch.cuh"

namespace csipm {

#define CSIPM_INST_R2(T, IN, OUT, MASK) \
    template cudaError_t launch_row2<T, IN, OUT, MASK>(int, int, const PassArgs<T>&, cudaStream_t);
CSIPM_FFT2_ROW_LIST32(CSIPM_INST_R2)
#undef CSIPM_INST_R2

}  // namespace csipm
