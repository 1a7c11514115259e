// Host-side FFT planning: radix factorisation and accurate twiddle tables.
#pragma once
#include <string>
#include <vector>

#include "fft_device.cuh"

namespace csipm {

// Factor L into stages: radix 8 first, then 4/2 for the rest of the power of
// two, then 5, 3, 7 and finally any other prime as a direct DFT stage.
bool make_fft_plan(int L, FftPlanDev* out, std::string* err);

// exp(-2*pi*i*e/L) for e = 0..L-1, rounded from long double.
void twiddle_table(int L, std::vector<double>* re_im);

// True when every stage of `pl` respects the per-thread register budget for
// `lines` interleaved lines processed by `nthreads` threads.
bool plan_fits(const FftPlanDev& pl, int lines, int nthreads);

}  // namespace csipm
