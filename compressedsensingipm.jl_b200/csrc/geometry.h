// Geometry of the Hermitian beta <-> spectrum packing and its per-position decode.
//
// The packing is the one of CompressedSensingIPM.jl (src/mapping_cpu.jl,
// src/mapping_cpu_kernels.jl): beta in R^N holds, in this order, the real
// "vertex" entries, then (re, im) pairs for edges, faces and the interior of the
// half spectrum, each pair scaled by sqrt(2).  Instead of the reference's chain
// of region tests per beta index, every spectrum position (i, j, k) is decoded
// here in O(1) from the class of each coordinate:
//
//   Z: x == 0      H: x == M      L: 1 <= x <= M-1      U: M+1 <= x <= N-1
//
// and yields the beta pair (re, im), the sign rule and whether DFT_to_beta reads
// this position ("source").  Positions with i > M1 (full spectrum only) are the
// conjugate of the mirror position, i.e. the same pair with the sign flipped.
//
// Value rules (bit-exact with src/mapping_cpu_kernels.jl):
//   VERT : v = (beta[re], +0)                         beta[re] = Re v
//   PLUS : v = (beta[re] + im*beta[im]) / sqrt(2)      beta[re] = sqrt2*Re v, beta[im] =  sqrt2*Im v
//   MINUS: v = (beta[re] - im*beta[im]) / sqrt(2)      beta[re] = sqrt2*Re v, beta[im] = -sqrt2*Im v
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define CSIPM_HD __host__ __device__ __forceinline__
#else
#define CSIPM_HD inline
#endif

namespace csipm {

enum MapKind : int { KIND_VERT = 0, KIND_PLUS = 1, KIND_MINUS = 2 };

struct MapEntry {
    int re;
    int im;
    int kind;
    int src;
};

struct Geom {
    int dim;
    int n1, n2, n3;
    int m1, m2, m3;
    int p1, p2, p3;
    int ld1;        // pitch of the spectrum along dim 1 (complex elements)
    int64_t N;      // n1*n2*n3
    int64_t Nh;     // (m1+1)*n2*n3
    int64_t NI;     // (m1-1)*n2*n3: interior half-spectrum positions (solver-order pairs)
    // 3D block offsets (0-based beta index where each region starts)
    int oE2, oE1;            // j-edges, i-edges (k-edges start at 8)
    int oFi, oFj, oFk, oC;   // faces i, faces j, faces k, interior
    int P23, P13, P12, P123;
    // 2D block offsets
    int o2E1, o2C, PP;
};

inline Geom make_geom(int dim, const int* n, int ld1) {
    Geom g{};
    g.dim = dim;
    g.n1 = n[0];
    g.n2 = dim >= 2 ? n[1] : 1;
    g.n3 = dim >= 3 ? n[2] : 1;
    g.m1 = g.n1 / 2; g.m2 = g.n2 / 2; g.m3 = g.n3 / 2;
    g.p1 = g.m1 - 1; g.p2 = g.m2 - 1; g.p3 = g.m3 - 1;
    g.ld1 = ld1;
    g.N = (int64_t)g.n1 * g.n2 * g.n3;
    g.Nh = (int64_t)(g.m1 + 1) * g.n2 * g.n3;
    g.NI = (int64_t)(g.m1 - 1) * g.n2 * g.n3;
    g.P23 = g.p2 * g.p3; g.P13 = g.p1 * g.p3; g.P12 = g.p1 * g.p2; g.P123 = g.p1 * g.p2 * g.p3;
    g.oE2 = 8 + 8 * g.p3;
    g.oE1 = g.oE2 + 8 * g.p2;
    g.oFi = g.oE1 + 8 * g.p1;
    g.oFj = g.oFi + 8 * g.P23;
    g.oFk = g.oFj + 8 * g.P13;
    g.oC = g.oFk + 8 * g.P12;
    g.PP = g.p1 * g.p2;
    g.o2E1 = 4 + 4 * g.p2;
    g.o2C = g.o2E1 + 4 * g.p1;
    return g;
}

// coordinate class: 0 = Z (x==0), 1 = H (x==M), 2 = L, 3 = U
CSIPM_HD int coord_class(int x, int M) {
    return x == 0 ? 0 : (x == M ? 1 : (x < M ? 2 : 3));
}

CSIPM_HD MapEntry flip_entry(MapEntry e) {
    if (e.kind == KIND_PLUS) e.kind = KIND_MINUS;
    else if (e.kind == KIND_MINUS) e.kind = KIND_PLUS;
    e.src = 0;
    return e;
}

CSIPM_HD MapEntry decode1(const Geom& g, int i) {
    MapEntry e;
    bool flip = false;
    if (i > g.m1) { i = g.n1 - i; flip = true; }
    if (i == 0) { e.re = 0; e.im = -1; e.kind = KIND_VERT; e.src = 1; }
    else if (i == g.m1) { e.re = 1; e.im = -1; e.kind = KIND_VERT; e.src = 1; }
    else { e.re = i + 1; e.im = g.m1 + i; e.kind = KIND_PLUS; e.src = 1; }
    return flip ? flip_entry(e) : e;
}

CSIPM_HD MapEntry decode2(const Geom& g, int i, int j) {
    MapEntry e;
    bool flip = false;
    if (i > g.m1) { i = g.n1 - i; j = (j == 0) ? 0 : g.n2 - j; flip = true; }
    const int ci = coord_class(i, g.m1), cj = coord_class(j, g.m2);
    if (ci <= 1) {
        if (cj <= 1) { e.re = 2 * ci + cj; e.im = -1; e.kind = KIND_VERT; e.src = 1; }
        else {
            const int base = 4 + 2 * ci * g.p2;
            if (cj == 2) { e.re = base + (j - 1); e.kind = KIND_PLUS; e.src = 1; }
            else { e.re = base + (g.n2 - j - 1); e.kind = KIND_MINUS; e.src = 0; }
            e.im = e.re + g.p2;
        }
    } else {
        const int ti = i - 1;
        if (cj <= 1) { e.re = g.o2E1 + 2 * cj * g.p1 + ti; e.im = e.re + g.p1; }
        else if (cj == 2) { e.re = g.o2C + (j - 1) * g.p1 + ti; e.im = e.re + g.PP; }
        else { e.re = g.o2C + 2 * g.PP + (j - g.m2 - 1) * g.p1 + ti; e.im = e.re + g.PP; }
        e.kind = KIND_PLUS; e.src = 1;
    }
    return flip ? flip_entry(e) : e;
}

CSIPM_HD MapEntry decode3(const Geom& g, int i, int j, int k) {
    MapEntry e;
    bool flip = false;
    if (i > g.m1) { i = g.n1 - i; j = (j == 0) ? 0 : g.n2 - j; k = (k == 0) ? 0 : g.n3 - k; flip = true; }
    const int ci = coord_class(i, g.m1), cj = coord_class(j, g.m2), ck = coord_class(k, g.m3);
    if (ci <= 1) {
        if (cj <= 1 && ck <= 1) {
            e.re = 4 * ci + 2 * cj + ck; e.im = -1; e.kind = KIND_VERT; e.src = 1;
        } else if (cj <= 1) {                   // edge along k
            const int base = 8 + 2 * (2 * ci + cj) * g.p3;
            if (ck == 2) { e.re = base + (k - 1); e.kind = KIND_PLUS; e.src = 1; }
            else { e.re = base + (g.n3 - k - 1); e.kind = KIND_MINUS; e.src = 0; }
            e.im = e.re + g.p3;
        } else if (ck <= 1) {                   // edge along j
            const int base = g.oE2 + 2 * (2 * ci + ck) * g.p2;
            if (cj == 2) { e.re = base + (j - 1); e.kind = KIND_PLUS; e.src = 1; }
            else { e.re = base + (g.n2 - j - 1); e.kind = KIND_MINUS; e.src = 0; }
            e.im = e.re + g.p2;
        } else {                                // face i
            const int o = g.oFi + 4 * ci * g.P23;
            if (ck == 2) {
                e.re = (cj == 2) ? o + (k - 1) * g.p2 + (j - 1)
                                 : o + 2 * g.P23 + (k - 1) * g.p2 + (j - g.m2 - 1);
                e.kind = KIND_PLUS; e.src = 1;
            } else {
                e.re = (cj == 2) ? o + 2 * g.P23 + (g.n3 - k - 1) * g.p2 + (g.m2 - j - 1)
                                 : o + (g.n3 - k - 1) * g.p2 + (g.n2 - j - 1);
                e.kind = KIND_MINUS; e.src = 0;
            }
            e.im = e.re + g.P23;
        }
    } else {
        const int ti = i - 1, tm = g.m1 - i - 1;
        if (cj <= 1 && ck <= 1) {               // edge along i
            e.re = g.oE1 + 2 * (2 * cj + ck) * g.p1 + ti; e.im = e.re + g.p1; e.kind = KIND_PLUS;
        } else if (cj <= 1) {                   // face j
            const int o = g.oFj + 4 * cj * g.P13;
            if (ck == 2) { e.re = o + (k - 1) * g.p1 + ti; e.kind = KIND_PLUS; }
            else { e.re = o + 2 * g.P13 + (g.n3 - k - 1) * g.p1 + tm; e.kind = KIND_MINUS; }
            e.im = e.re + g.P13;
        } else if (ck <= 1) {                   // face k
            const int o = g.oFk + 4 * ck * g.P12;
            if (cj == 2) { e.re = o + (j - 1) * g.p1 + ti; e.kind = KIND_PLUS; }
            else { e.re = o + 2 * g.P12 + (g.n2 - j - 1) * g.p1 + tm; e.kind = KIND_MINUS; }
            e.im = e.re + g.P12;
        } else {                                // interior
            if (cj == 2 && ck == 2) {
                e.re = g.oC + (k - 1) * g.P12 + (j - 1) * g.p1 + ti; e.kind = KIND_PLUS;
            } else if (cj == 3 && ck == 3) {
                e.re = g.oC + 2 * g.P123 + (g.n3 - k - 1) * g.P12 + (g.n2 - j - 1) * g.p1 + tm; e.kind = KIND_MINUS;
            } else if (cj == 3) {
                e.re = g.oC + 4 * g.P123 + (k - 1) * g.P12 + (j - g.m2 - 1) * g.p1 + ti; e.kind = KIND_PLUS;
            } else {
                e.re = g.oC + 6 * g.P123 + (g.n3 - k - 1) * g.P12 + (g.m2 - j - 1) * g.p1 + tm; e.kind = KIND_MINUS;
            }
            e.im = e.re + g.P123;
        }
        e.src = 1;
    }
    return flip ? flip_entry(e) : e;
}

// Decode for an interior dim-1 position (1 <= i <= M1-1, half spectrum), the
// case of all but two of every M1+1 positions: no mirror flip, no vertex,
// edge-along-k, edge-along-j or face-i branches.
CSIPM_HD MapEntry decode_interior(const Geom& g, int i, int j, int k) {
    MapEntry e;
    const int ti = i - 1, tm = g.m1 - i - 1;
    e.src = 1;
    if (g.dim == 2) {
        const int cj = coord_class(j, g.m2);
        e.kind = KIND_PLUS;
        if (cj <= 1) { e.re = g.o2E1 + 2 * cj * g.p1 + ti; e.im = e.re + g.p1; }
        else if (cj == 2) { e.re = g.o2C + (j - 1) * g.p1 + ti; e.im = e.re + g.PP; }
        else { e.re = g.o2C + 2 * g.PP + (j - g.m2 - 1) * g.p1 + ti; e.im = e.re + g.PP; }
        return e;
    }
    if (g.dim == 1) { e.re = i + 1; e.im = g.m1 + i; e.kind = KIND_PLUS; return e; }
    const int cj = coord_class(j, g.m2), ck = coord_class(k, g.m3);
    if (cj <= 1 && ck <= 1) {
        e.re = g.oE1 + 2 * (2 * cj + ck) * g.p1 + ti; e.im = e.re + g.p1; e.kind = KIND_PLUS;
    } else if (cj <= 1) {
        const int o = g.oFj + 4 * cj * g.P13;
        if (ck == 2) { e.re = o + (k - 1) * g.p1 + ti; e.kind = KIND_PLUS; }
        else { e.re = o + 2 * g.P13 + (g.n3 - k - 1) * g.p1 + tm; e.kind = KIND_MINUS; }
        e.im = e.re + g.P13;
    } else if (ck <= 1) {
        const int o = g.oFk + 4 * ck * g.P12;
        if (cj == 2) { e.re = o + (j - 1) * g.p1 + ti; e.kind = KIND_PLUS; }
        else { e.re = o + 2 * g.P12 + (g.n2 - j - 1) * g.p1 + tm; e.kind = KIND_MINUS; }
        e.im = e.re + g.P12;
    } else if (cj == 2 && ck == 2) {
        e.re = g.oC + (k - 1) * g.P12 + (j - 1) * g.p1 + ti; e.im = e.re + g.P123; e.kind = KIND_PLUS;
    } else if (cj == 3 && ck == 3) {
        e.re = g.oC + 2 * g.P123 + (g.n3 - k - 1) * g.P12 + (g.n2 - j - 1) * g.p1 + tm; e.im = e.re + g.P123; e.kind = KIND_MINUS;
    } else if (cj == 3) {
        e.re = g.oC + 4 * g.P123 + (k - 1) * g.P12 + (j - g.m2 - 1) * g.p1 + ti; e.im = e.re + g.P123; e.kind = KIND_PLUS;
    } else {
        e.re = g.oC + 6 * g.P123 + (g.n3 - k - 1) * g.P12 + (g.m2 - j - 1) * g.p1 + tm; e.im = e.re + g.P123; e.kind = KIND_MINUS;
    }
    return e;
}

CSIPM_HD MapEntry decode(const Geom& g, int i, int j, int k) {
    return g.dim == 3 ? decode3(g, i, j, k) : (g.dim == 2 ? decode2(g, i, j) : decode1(g, i));
}

// ---------------------------------------------------------------- solver order
// The interior-point solve keeps its beta-space vectors in a "solver order"
// that follows the half spectrum instead of the reference packing:
//
//   pairs: for 1 <= i <= M1-1 (every such position is a source of a pair),
//          x[2q], x[2q+1] with q = (k*N2 + j)*(M1-1) + (i-1) hold
//          sqrt2*(Re X, Im X) = (beta[re], +-beta[im]), the sign of the
//          reference's MINUS pairs folded in;
//   tail:  the 2*N2*N3 entries of the planes i = 0 and i = M1 (vertices,
//          edges along j and k, faces i) in reference order, from 2*NI on.
//
// A gather is then one 16-byte load per spectrum position and a scatter one
// 16-byte store, with the same (i, j, k) walk as the spectrum itself.  The map
// is a signed permutation; the LASSO objective, the split-variable bounds and
// every step of the interior-point method commute with it, so the solve in
// solver order follows the same iterates (up to the order of floating-point
// sums) and its result is mapped back to reference order at the end.
CSIPM_HD int64_t sol_pair(const Geom& g, int i, int j, int k) {
    return ((int64_t)k * g.n2 + j) * (g.m1 - 1) + (i - 1);
}

// solver-order index of a plane entry (reference index `ref`, i = 0 or M1)
CSIPM_HD int64_t sol_tail(const Geom& g, int ref) {
    const int64_t t = (g.dim == 3 && ref >= g.oFi) ? (int64_t)ref - g.oFi + g.oE1 : (int64_t)ref;
    return 2 * g.NI + t;
}

// reference index of tail entry t (0 <= t < 2*N2*N3)
CSIPM_HD int64_t sol_tail_ref(const Geom& g, int64_t t) {
    return (g.dim == 3 && t >= g.oE1) ? t - g.oE1 + g.oFi : t;
}

}  // namespace csipm
