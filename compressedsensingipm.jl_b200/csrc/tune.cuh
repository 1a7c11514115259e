// Per-size autotuner of the FFT passes.
//
// For a new (precision, dims, mask) the handle times each candidate launch
// configuration of its passes on its own spectrum buffer (CUDA events on the
// handle's stream, one warm launch, best of TUNE_REPS) and keeps the fastest:
//
//   dim-3 lines:  two-level register kernel (when the length has a pair)
//                 or the Stockham kernel with 2/4/8(/16 in FP32) lines per CTA
//   dim-2 lines:  Stockham lines per CTA when the length has no pair (with a
//                 pair the two-level kernel stays: the solver-order gather and
//                 scatter need it)
//   dim-1 rows:   two-level row kernel (pair) or Stockham with 1..16 rows per CTA
//
// Results are cached per process, so every later handle of the same size
// starts with the tuned configuration at no cost.  When the environment
// variable CSIPM_TUNE_CACHE names a file, the cache persists across
// processes: the file's choices are read at the first tuning, and every new
// choice is appended to it as one JSON object per line,
//   {"elem": 4, "dim": 3, "n": [320, 320, 320], "masked": 1,
//    "s3_two": 1, "s3_tb": 0, "s2_tb": 0, "row_two": 1, "row_rb": 0}
#pragma once
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>
#include <tuple>

#include "internal.h"

namespace csipm_internal {

struct TuneChoice {
    int s3_two = 1, s3_tb = 0;     // 1: two-level; else Stockham tb (0: the heuristic's)
    int s2_tb = 0;
    int row_two = 1, row_rb = 0;
};

constexpr int TUNE_REPS = 3;
// a candidate replaces the incumbent only when it is this much faster
// (timing noise must not flip between kernels of equal speed)
constexpr float TUNE_MARGIN = 0.95f;

using TuneKey = std::tuple<int, int, int, int, int, int>;   // sizeof(T), dim, n1, n2, n3, masked

inline std::mutex& tune_mu() {
    static std::mutex m;
    return m;
}
inline std::map<TuneKey, TuneChoice>& tune_cache() {
    static std::map<TuneKey, TuneChoice> c;
    return c;
}

// CSIPM_TUNE_CACHE: "" when unset
inline const std::string& tune_cache_path() {
    static const std::string p = [] {
        const char* e = std::getenv("CSIPM_TUNE_CACHE");
        return std::string(e ? e : "");
    }();
    return p;
}

// Reads the persisted choices once (tune_mu held); lines that do not parse are skipped.
inline void tune_cache_load() {
    static bool loaded = false;
    if (loaded) return;
    loaded = true;
    const std::string& path = tune_cache_path();
    if (path.empty()) return;
    FILE* f = std::fopen(path.c_str(), "r");
    if (!f) return;
    char line[512];
    while (std::fgets(line, sizeof(line), f)) {
        int elem, dim, n1, n2, n3, masked;
        TuneChoice c;
        if (std::sscanf(line,
                        " {\"elem\": %d, \"dim\": %d, \"n\": [%d, %d, %d], \"masked\": %d, \"s3_two\": %d, "
                        "\"s3_tb\": %d, \"s2_tb\": %d, \"row_two\": %d, \"row_rb\": %d}",
                        &elem, &dim, &n1, &n2, &n3, &masked, &c.s3_two, &c.s3_tb, &c.s2_tb, &c.row_two,
                        &c.row_rb) == 11)
            tune_cache()[TuneKey{elem, dim, n1, n2, n3, masked}] = c;
    }
    std::fclose(f);
}

// Appends one choice to the persisted cache (tune_mu held).
inline void tune_cache_append(const TuneKey& k, const TuneChoice& c) {
    const std::string& path = tune_cache_path();
    if (path.empty()) return;
    FILE* f = std::fopen(path.c_str(), "a");
    if (!f) return;
    std::fprintf(f,
                 "{\"elem\": %d, \"dim\": %d, \"n\": [%d, %d, %d], \"masked\": %d, \"s3_two\": %d, "
                 "\"s3_tb\": %d, \"s2_tb\": %d, \"row_two\": %d, \"row_rb\": %d}\n",
                 std::get<0>(k), std::get<1>(k), std::get<2>(k), std::get<3>(k), std::get<4>(k), std::get<5>(k),
                 c.s3_two, c.s3_tb, c.s2_tb, c.row_two, c.row_rb);
    std::fclose(f);
}

// Stockham strided configuration with a forced number of lines per CTA
template <typename T>
bool strided_cfg_tb(const FftOperator<T>& op, const FftPlanDev& pl, int Ltab, int n_lines, int n_outer, int tb,
                    PassCfg* cfg) {
    using C = cplx_t<T>;
    const size_t data = 3 * (size_t)pl.L * sizeof(C) * tb;
    if (data > FftOperator<T>::smem_limit() || data > 96 * 1024) return false;
    cfg->tb = tb;
    cfg->tbp = tb;
    cfg->threads = 256;
    cfg->pp = 1;
    const size_t tws = (size_t)Ltab * sizeof(C);
    cfg->tw_in_smem = (data + tws <= FftOperator<T>::smem_limit() && tws <= 32 * 1024) ? 1 : 0;
    cfg->smem = data + (cfg->tw_in_smem ? tws : 0);
    cfg->tiles = ((n_lines + tb - 1) / tb) * n_outer;
    cfg->grid = dim3(cfg->tiles, 1, 1);
    return true;
}

// Stockham persistent row configuration with a forced number of rows per CTA
template <typename T>
bool row_cfg_rb(const FftOperator<T>& op, int nrows, int rb, PassCfg* cfg) {
    using C = cplx_t<T>;
    const int M = op.g.m1;
    if (rb > nrows) return false;
    const int tbp = rb > 1 ? rb + 1 : 1;
    const size_t one = (size_t)(M + 1) * tbp * sizeof(C);
    if (3 * one > FftOperator<T>::smem_limit() || 3 * one > 96 * 1024) return false;
    const size_t tws = (size_t)op.g.n1 * sizeof(C);
    cfg->pp = 1;
    cfg->tb = rb;
    cfg->tbp = tbp;
    cfg->threads = 256;
    cfg->tw_in_smem = (3 * one + tws <= FftOperator<T>::smem_limit() && tws <= 32 * 1024) ? 1 : 0;
    cfg->smem = 3 * one + (cfg->tw_in_smem ? tws : 0);
    cfg->tiles = (nrows + rb - 1) / rb;
    cfg->grid = dim3(cfg->tiles, 1, 1);
    return true;
}

template <typename T, class F>
float tune_time(cudaStream_t st, cudaEvent_t e0, cudaEvent_t e1, F&& launch) {
    if (launch() != cudaSuccess) {
        cudaGetLastError();
        return 1e30f;
    }
    float best = 1e30f;
    for (int r = 0; r < TUNE_REPS; ++r) {
        cudaEventRecord(e0, st);
        if (launch() != cudaSuccess) {
            cudaGetLastError();
            return 1e30f;
        }
        cudaEventRecord(e1, st);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        best = std::min(best, ms);
    }
    return best;
}

template <typename T>
void apply_choice(FftOperator<T>& op, const TuneChoice& c) {
    const Geom& g = op.g;
    if (g.dim == 3) {
        if (!c.s3_two) op.s3_A = op.s3_B = 0;
        if (c.s3_tb) strided_cfg_tb(op, op.plan3, g.n3, g.m1 + 1, g.n2, c.s3_tb, &op.s3_cfg);
    }
    if (g.dim >= 2 && c.s2_tb) strided_cfg_tb(op, op.plan2, g.n2, g.m1 + 1, g.dim == 3 ? g.n3 : 1, c.s2_tb, &op.s2_cfg);
    if (g.dim >= 2) {
        if (!c.row_two) op.r_A = op.r_B = 0;
        if (c.row_rb) row_cfg_rb(op, g.n2 * g.n3, c.row_rb, &op.row_cfg);
    }
}

// Tunes op (2D/3D; 1D keeps its heuristic) on stream st; op.spec holds scratch.
template <typename T>
void autotune(FftOperator<T>& op, cudaStream_t st) {
    const Geom& g = op.g;
    if (g.dim < 2) return;
    const TuneKey key{(int)sizeof(T), g.dim, g.n1, g.n2, g.n3, op.maskw ? 1 : 0};
    {
        std::lock_guard<std::mutex> lk(tune_mu());
        tune_cache_load();
        auto it = tune_cache().find(key);
        if (it != tune_cache().end()) {
            apply_choice(op, it->second);
            return;
        }
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaMemsetAsync(op.spec, 0, sizeof(cplx_t<T>) * (size_t)g.ld1 * g.n2 * g.n3, st);
    EpiStore<double> none{nullptr};
    TuneChoice best;
    const int tbs[4] = {2, 4, 8, 16};
    const int max_tb = sizeof(T) == 8 ? 8 : 16;
    // dim-3 lines
    if (g.dim == 3) {
        const int A = op.s3_A, B = op.s3_B;
        const PassCfg keep = op.s3_cfg;
        float t_best = 1e30f;
        if (A) {
            t_best = tune_time<T>(st, e0, e1, [&] {
                return run_strided<T, true, IN_SPEC, OUT_SPEC>(op, 3, op.strided_args(3), (const double*)nullptr, none, st);
            });
        }
        best.s3_two = A ? 1 : 0;
        op.s3_A = op.s3_B = 0;
        for (int tb : tbs) {
            if (tb > max_tb) continue;
            PassCfg c;
            if (!strided_cfg_tb(op, op.plan3, g.n3, g.m1 + 1, g.n2, tb, &c)) continue;
            op.s3_cfg = c;
            const float t = tune_time<T>(st, e0, e1, [&] {
                return run_strided<T, true, IN_SPEC, OUT_SPEC>(op, 3, op.strided_args(3), (const double*)nullptr, none, st);
            });
            if (t < TUNE_MARGIN * t_best) { t_best = t; best.s3_two = 0; best.s3_tb = tb; }
        }
        op.s3_A = A;
        op.s3_B = B;
        op.s3_cfg = keep;
    }
    // dim-2 lines without a two-level pair
    if (!op.s2_A) {
        const PassCfg keep = op.s2_cfg;
        float t_best = tune_time<T>(st, e0, e1, [&] {
            return run_strided<T, true, IN_SPEC, OUT_SPEC>(op, 2, op.strided_args(2), (const double*)nullptr, none, st);
        });
        for (int tb : tbs) {
            if (tb > max_tb) continue;
            PassCfg c;
            if (!strided_cfg_tb(op, op.plan2, g.n2, g.m1 + 1, g.dim == 3 ? g.n3 : 1, tb, &c)) continue;
            op.s2_cfg = c;
            const float t = tune_time<T>(st, e0, e1, [&] {
                return run_strided<T, true, IN_SPEC, OUT_SPEC>(op, 2, op.strided_args(2), (const double*)nullptr, none, st);
            });
            if (t < TUNE_MARGIN * t_best) { t_best = t; best.s2_tb = tb; }
        }
        op.s2_cfg = keep;
    }
    // dim-1 rows (persistent Stockham candidates only when the heuristic's row
    // configuration is the persistent one)
    {
        const int A = op.r_A, B = op.r_B;
        const PassCfg keep = op.row_cfg;
        const bool mask = op.maskw != nullptr;
        PassArgs<T> ra = op.row_args(1.0, nullptr, nullptr);
        auto row = [&] {
            return mask ? run_row<T, IN_SPEC, OUT_SPEC, true>(op, ra, (const double*)nullptr, none, st)
                        : run_row<T, IN_SPEC, OUT_SPEC, false>(op, ra, (const double*)nullptr, none, st);
        };
        float t_best = tune_time<T>(st, e0, e1, row);
        best.row_two = A ? 1 : 0;
        if (keep.pp) {
            op.r_A = op.r_B = 0;
            for (int rb : {1, 2, 4, 8, 16}) {
                PassCfg c;
                if (!row_cfg_rb(op, g.n2 * g.n3, rb, &c)) continue;
                op.row_cfg = c;
                ra = op.row_args(1.0, nullptr, nullptr);
                const float t = tune_time<T>(st, e0, e1, row);
                if (t < TUNE_MARGIN * t_best) { t_best = t; best.row_two = 0; best.row_rb = rb; }
            }
        }
        op.r_A = A;
        op.r_B = B;
        op.row_cfg = keep;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    {
        std::lock_guard<std::mutex> lk(tune_mu());
        if (tune_cache().emplace(key, best).second) tune_cache_append(key, best);
    }
    apply_choice(op, best);
}

}  // namespace csipm_internal
