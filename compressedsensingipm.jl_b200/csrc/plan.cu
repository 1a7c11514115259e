#include "plan.h"

#include <cmath>

namespace csipm {

bool make_fft_plan(int L, FftPlanDev* out, std::string* err, int max_radix) {
    FftPlanDev p{};
    p.L = L;
    p.nst = 0;
    if (L < 1) {
        if (err) *err = "FFT length must be positive";
        return false;
    }
    if (max_radix > 8) {
        static const int cand[] = {32, 25, 20, 16, 15, 12, 10, 9, 8, 7, 6, 5, 4, 3, 2};
        int r = L;
        while (r > 1) {
            int pick = 0;
            for (int c : cand)
                if (c <= max_radix && r % c == 0) { pick = c; break; }
            if (!pick) {   // a prime > 7 (or a composite of them): smallest factor as a direct DFT
                pick = r;
                for (int f = 11; (long long)f * f <= r; f += 2)
                    if (r % f == 0) { pick = f; break; }
            }
            if (p.nst >= FFT_MAX_STAGES) {
                if (err) *err = "FFT length has too many prime factors";
                return false;
            }
            p.rad[p.nst++] = pick;
            r /= pick;
        }
        *out = p;
        return true;
    }
    int r = L;
    int twos = 0;
    while (r % 2 == 0) { r /= 2; ++twos; }
    auto push = [&](int radix) -> bool {
        if (p.nst >= FFT_MAX_STAGES) return false;
        p.rad[p.nst++] = radix;
        return true;
    };
    // 2^twos = 8^a * {1, 4*4 (for 2^4 -> 16 when rem 1), 4 (rem 2)} ; a lone 2 only for L=2
    int rem = twos % 3, a = twos / 3;
    if (rem == 1 && a >= 1) { a -= 1; rem = 4; }   // 8*2 -> 4*4
    for (int i = 0; i < a; ++i) if (!push(8)) goto too_many;
    if (rem == 1) { if (!push(2)) goto too_many; }
    else if (rem == 2) { if (!push(4)) goto too_many; }
    else if (rem == 4) { if (!push(4) || !push(4)) goto too_many; }
    for (int f : {5, 3, 7}) {
        while (r % f == 0) { if (!push(f)) goto too_many; r /= f; }
    }
    for (int f = 11; r > 1; f += 2) {
        while (r % f == 0) { if (!push(f)) goto too_many; r /= f; }
        if ((long long)f * f > r && r > 1) { if (!push(r)) goto too_many; r = 1; }
    }
    *out = p;
    return true;
too_many:
    if (err) *err = "FFT length has too many prime factors";
    return false;
}

bool plan_fits(const FftPlanDev& pl, int lines, int nthreads) {
    const long long total = (long long)lines * pl.L;
    for (int s = 0; s < pl.nst; ++s) {
        const int R = pl.rad[s];
        long long items;
        long long cap;
        switch (R) {
            case 2: cap = MaxItems<2>::v; break;
            case 3: cap = MaxItems<3>::v; break;
            case 4: cap = MaxItems<4>::v; break;
            case 5: cap = MaxItems<5>::v; break;
            case 7: cap = MaxItems<7>::v; break;
            case 8: cap = MaxItems<8>::v; break;
            default: cap = GENERIC_MAX_ITEMS; break;
        }
        if (R == 2 || R == 3 || R == 4 || R == 5 || R == 7 || R == 8)
            items = (total / R + nthreads - 1) / nthreads;
        else
            items = (total + nthreads - 1) / nthreads;
        if (items > cap) return false;
    }
    return true;
}

}  // namespace csipm
