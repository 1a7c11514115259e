// Host-side FFT planning: radix factorisation.  (Twiddle tables are built on
// the device: launch_twiddles in operator.cuh.)
#pragma once
#include <string>
#include <vector>

#include "fft_device.cuh"

namespace csipm {

// Factor L into stages.  max_radix <= 8: radix 8 first, then 4/2 for the rest
// of the power of two, then 5, 3, 7 (the register-staged in-place engine).
// Larger max_radix: greedy largest-first over the composite register radices
// {32, 25, 20, 16, 15, 12, 10, 9, 8, 7, 6, 5, 4, 3, 2} up to max_radix, which
// cuts the number of shared-memory round trips (320 = 20*16, 160 = 20*8).
// Any remaining prime becomes a direct-DFT stage.
bool make_fft_plan(int L, FftPlanDev* out, std::string* err, int max_radix = 8);

// True when every stage of `pl` respects the per-thread register budget for
// `lines` interleaved lines processed by `nthreads` threads.
bool plan_fits(const FftPlanDev& pl, int lines, int nthreads);

}  // namespace csipm
