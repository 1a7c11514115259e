// C ABI (include/csipm.h), part 3: the bit-exact beta <-> DFT maps.
#include "internal.h"

namespace {

constexpr double SQRT2_EXACT = 1.4142135623730951;

// ------------------------------------------------------------------ map kernels
// Bit-exact beta_to_DFT (src/mapping_cpu_kernels.jl:354-738): IEEE division by
// sqrt(2), Julia's signed-zero rule for a +/- im*b (real part a +/- copysign(0,b)).
__global__ void map_b2d_kernel(Geom g, int ni, const double* __restrict__ beta, double2* __restrict__ v) {
    const long long total = (long long)ni * g.n2 * g.n3;
    CSIPM_GRID_LOOP(idx, total) {
        const int i = (int)(idx % ni);
        const long long rest = idx / ni;
        const int j = (int)(rest % g.n2), k = (int)(rest / g.n2);
        const MapEntry e = decode(g, i, j, k);
        double re, im;
        if (e.kind == KIND_VERT) {
            re = beta[e.re];
            im = 0.0;
        } else {
            const double a = beta[e.re], b = beta[e.im];
            if (e.kind == KIND_PLUS) {
                re = __ddiv_rn(__dadd_rn(a, copysign(0.0, b)), SQRT2_EXACT);
                im = __ddiv_rn(b, SQRT2_EXACT);
            } else {
                re = __ddiv_rn(__dsub_rn(a, copysign(0.0, b)), SQRT2_EXACT);
                im = __ddiv_rn(-b, SQRT2_EXACT);
            }
        }
        v[idx] = make_double2(re, im);
    }
}

// Bit-exact DFT_to_beta (src/mapping_cpu_kernels.jl:2-351): reads the half spectrum only.
__global__ void map_d2b_kernel(Geom g, const double2* __restrict__ v, double* __restrict__ beta) {
    const int ni = g.m1 + 1;
    const long long total = (long long)ni * g.n2 * g.n3;
    CSIPM_GRID_LOOP(idx, total) {
        const int i = (int)(idx % ni);
        const long long rest = idx / ni;
        const int j = (int)(rest % g.n2), k = (int)(rest / g.n2);
        const MapEntry e = decode(g, i, j, k);
        if (!e.src) continue;
        const double2 z = v[i + (long long)g.ld1 * (j + (long long)g.n2 * k)];
        if (e.kind == KIND_VERT) {
            beta[e.re] = z.x;
        } else {
            beta[e.re] = __dmul_rn(SQRT2_EXACT, z.x);
            beta[e.im] = __dmul_rn(e.kind == KIND_PLUS ? SQRT2_EXACT : -SQRT2_EXACT, z.y);
        }
    }
}


}  // namespace

extern "C" {

int csipm_beta_to_dft(int dim, const int* size, int rdft, const double* beta, double* v, void* stream) {
    csipm_handle h = nullptr;
    std::string err;
    int status = 0;
    if (!valid_dims(dim, size, &err, &status)) return fail(h, status, err);
    if (!beta || !v) return fail(h, CSIPM_ERR_INVALID, "null argument");
    int n[3] = {size[0], dim >= 2 ? size[1] : 1, dim >= 3 ? size[2] : 1};
    const int ni = rdft ? n[0] / 2 + 1 : n[0];
    Geom g = make_geom(dim, n, ni);
    const long long total = (long long)ni * g.n2 * g.n3;
    map_b2d_kernel<<<ew_blocks(total), EW_THREADS, 0, (cudaStream_t)stream>>>(g, ni, beta, reinterpret_cast<double2*>(v));
    CK(cudaGetLastError());
    return CSIPM_OK;
}

int csipm_dft_to_beta(int dim, const int* size, int ld1, const double* v, double* beta, void* stream) {
    csipm_handle h = nullptr;
    std::string err;
    int status = 0;
    if (!valid_dims(dim, size, &err, &status)) return fail(h, status, err);
    if (!beta || !v) return fail(h, CSIPM_ERR_INVALID, "null argument");
    if (ld1 < size[0] / 2 + 1) return fail(h, CSIPM_ERR_INVALID, "ld1 must be >= N1/2+1");
    int n[3] = {size[0], dim >= 2 ? size[1] : 1, dim >= 3 ? size[2] : 1};
    Geom g = make_geom(dim, n, ld1);
    map_d2b_kernel<<<ew_blocks(g.Nh), EW_THREADS, 0, (cudaStream_t)stream>>>(g, reinterpret_cast<const double2*>(v), beta);
    CK(cudaGetLastError());
    return CSIPM_OK;
}

}  // extern "C"
