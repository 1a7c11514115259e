#include "plan.h"

#include <cmath>
#include <list>
#include <memory>
#include <mutex>

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

// exp(-2*pi*i*num/L) in long double: the angle is reduced to the first
// octant (exact rational arithmetic on num/L) and rebuilt by symmetry.
static void root_ld(long long num, int L, long double* c, long double* s) {
    const long double twopi = 6.283185307179586476925286766559005768L;
    const long long n8 = 8LL * num;   // octant index = floor(8*num/L)
    const int oct = (int)(n8 / L);
    const long double frac = (long double)(n8 - (long long)oct * L) / (long double)L;   // in [0,1)
    const long double th = frac * (twopi / 8.0L);                                         // [0, pi/4)
    const long double cs = cosl(th), sn = sinl(th);
    const long double h = 0.70710678118654752440084436210484903928L;
    switch (oct) {
        case 0: *c = cs; *s = sn; break;
        case 1: *c = h * (cs - sn); *s = h * (cs + sn); break;
        case 2: *c = -sn; *s = cs; break;
        case 3: *c = -h * (cs + sn); *s = h * (cs - sn); break;
        case 4: *c = -cs; *s = -sn; break;
        case 5: *c = -h * (cs - sn); *s = -h * (cs + sn); break;
        case 6: *c = sn; *s = -cs; break;
        default: *c = h * (cs + sn); *s = -h * (cs - sn); break;
    }
}

// Fills the table from its first octant with exact symmetries of the roots
// of unity (sign changes and swaps only, so every entry keeps the accuracy
// of a directly rounded one):
//   e in (L/8, L/4):  W^e = (-Im W^(L/4-e), -Re W^(L/4-e))   (reflection, 8 | L)
//   e in [L/4, L/2]:  W^e = -i W^(e-L/4)                       (quarter turn, 4 | L)
//   e in (L/2, L):    W^e = conj W^(L-e)                       (conjugation)
// Lengths without those factors compute the remaining range directly.
static void build_table(int L, std::vector<double>& t) {
    t.resize(2 * (size_t)L);
    auto direct = [&](int e) {
        long double c, s;
        root_ld(e, L, &c, &s);
        t[2 * (size_t)e] = (double)c;
        t[2 * (size_t)e + 1] = (double)(-s);   // exp(-i*angle)
    };
    const bool q4 = L % 4 == 0, q8 = L % 8 == 0;
    const int half = L / 2;               // e <= half computed (or derived) first
    const int quarter = q4 ? L / 4 : half;
    const int eighth = q8 ? L / 8 : quarter;
    for (int e = 0; e <= eighth && e < L; ++e) direct(e);
    for (int e = eighth + 1; e < quarter; ++e) {
        if (q8) {
            const size_t m = (size_t)(L / 4 - e);
            t[2 * (size_t)e] = -t[2 * m + 1];
            t[2 * (size_t)e + 1] = -t[2 * m];
        } else {
            direct(e);
        }
    }
    for (int e = quarter; e <= half && e < L; ++e) {
        if (q4) {
            const size_t m = (size_t)(e - L / 4);
            t[2 * (size_t)e] = t[2 * m + 1];
            t[2 * (size_t)e + 1] = -t[2 * m];
        } else {
            direct(e);
        }
    }
    for (int e = half + 1; e < L; ++e) {
        const size_t m = (size_t)(L - e);
        t[2 * (size_t)e] = t[2 * m];
        t[2 * (size_t)e + 1] = -t[2 * m + 1];
    }
}

void twiddle_table(int L, std::vector<double>* re_im) {
    // process-wide cache of recent tables: the FP64 and FP32 operators of a
    // handle, and handles of repeated sizes, share one computation
    constexpr size_t CACHE_BYTES = 64u << 20;
    static std::mutex mu;
    static std::list<std::pair<int, std::shared_ptr<const std::vector<double>>>> cache;   // most recent first
    {
        std::lock_guard<std::mutex> lk(mu);
        for (auto it = cache.begin(); it != cache.end(); ++it) {
            if (it->first == L) {
                cache.splice(cache.begin(), cache, it);
                *re_im = *cache.front().second;
                return;
            }
        }
    }
    auto t = std::make_shared<std::vector<double>>();
    build_table(L, *t);
    *re_im = *t;
    std::lock_guard<std::mutex> lk(mu);
    cache.emplace_front(L, t);
    size_t bytes = 0;
    for (auto it = cache.begin(); it != cache.end();) {
        bytes += sizeof(double) * it->second->size();
        if (bytes > CACHE_BYTES && it != cache.begin()) it = cache.erase(it);
        else ++it;
    }
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
