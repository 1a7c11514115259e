/*
 * ORACLE — test infrastructure only.  Nothing in the product library links,
 * loads or calls this file; only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py use it, as the checker.
 *
 * CPU restatement of the beta <-> DFT packing of CompressedSensingIPM.jl in
 * two independent forms, both following the reference line by line:
 *
 *   orc_loops_*  : the region loops of   src/mapping_cpu.jl      (active CPU path)
 *   orc_kern_*   : the per-index decode of src/mapping_cpu_kernels.jl
 *                  (one scalar "kernel" per output index; the bit-exact target)
 *
 * Arrays are column-major (dim 1 fastest) like Julia.  Complex arrays are
 * interleaved (re, im) doubles.  `ld1` is the first-dimension extent of the
 * complex array: M1+1 for a half spectrum (rdft=true), N1 for a full one.
 * All index arithmetic below is 1-based to mirror the Julia sources.
 *
 * Julia scalar semantics restated exactly (they decide signed zeros):
 *   a + im*b      -> (a + copysign(0,b), b)      [im*b = (b*false, b*true);
 *                                                  Bool*Float: false*b = copysign(0,b)]
 *   a - im*b      -> (a - copysign(0,b), -b)
 *   z / sqrt(2)   -> (re/sqrt2, im/sqrt2)         (IEEE division, not a reciprocal)
 *   conj(z)       -> (re, -im)
 *   v[..] = real  -> (real, +0.0)
 *   sqrt(2)*x, -sqrt(2)*x  -> IEEE products
 */
#include <math.h>
#include <stdint.h>

#define SQRT2 1.4142135623730951

typedef struct { double re, im; } cplx;

static inline cplx jl_plus_im(double a, double b) {   /* a + im*b */
    cplx z; z.re = a + copysign(0.0, b); z.im = b; return z;
}
static inline cplx jl_minus_im(double a, double b) {  /* a - im*b */
    cplx z; z.re = a - copysign(0.0, b); z.im = -b; return z;
}
static inline cplx jl_div_sqrt2(cplx z) { z.re = z.re / SQRT2; z.im = z.im / SQRT2; return z; }
static inline cplx jl_conj(cplx z) { z.im = -z.im; return z; }
static inline cplx jl_real(double a) { cplx z; z.re = a; z.im = 0.0; return z; }

/* 1-based accessors */
#define B(l)          beta[(l) - 1]
#define VIDX1(i)      ((int64_t)(i) - 1)
#define VIDX2(i, j)   (((int64_t)(i) - 1) + (int64_t)ld1 * ((int64_t)(j) - 1))
#define VIDX3(i, j, k) (((int64_t)(i) - 1) + (int64_t)ld1 * (((int64_t)(j) - 1) + (int64_t)N2 * ((int64_t)(k) - 1)))

static inline cplx getc(const double *v, int64_t idx) { cplx z; z.re = v[2 * idx]; z.im = v[2 * idx + 1]; return z; }
static inline void setc(double *v, int64_t idx, cplx z) { v[2 * idx] = z.re; v[2 * idx + 1] = z.im; }

/* ======================================================================== */
/*  src/mapping_cpu.jl : DFT_to_beta_{1,2,3}d!  (lines 2-186)                */
/* ======================================================================== */

/* src/mapping_cpu.jl:2-12 */
void orc_loops_dft_to_beta_1d(double *beta, const double *v, int N, int ld1) {
    (void)ld1;
    int M = N / 2;
    B(1) = getc(v, VIDX1(1)).re;
    B(2) = getc(v, VIDX1(M + 1)).re;
    for (int i = 2; i <= M; i++) {
        cplx z = getc(v, VIDX1(i));
        B(i + 1) = SQRT2 * z.re;
        B(i + M) = SQRT2 * z.im;
    }
}

/* src/mapping_cpu.jl:14-57 */
void orc_loops_dft_to_beta_2d(double *beta, const double *v, int N1, int N2, int ld1) {
    int M1 = N1 / 2, M2 = N2 / 2, P1 = M1 - 1, P2 = M2 - 1, PP = P1 * P2;
#define V2(i, j) getc(v, VIDX2(i, j))
    B(1) = V2(1, 1).re;
    B(2) = V2(1, M2 + 1).re;
    B(3) = V2(M1 + 1, 1).re;
    B(4) = V2(M1 + 1, M2 + 1).re;
    int index = 4;
    for (int l = index + 1; l <= index + P2; l++) {
        int t = l - index + 1;
        B(l) = SQRT2 * V2(1, t).re;
        B(l + P2) = SQRT2 * V2(1, t).im;
        B(l + 2 * P2) = SQRT2 * V2(M1 + 1, t).re;
        B(l + 3 * P2) = SQRT2 * V2(M1 + 1, t).im;
    }
    index = index + 4 * P2;
    for (int l = index + 1; l <= index + P1; l++) {
        int t = l - index + 1;
        B(l) = SQRT2 * V2(t, 1).re;
        B(l + P1) = SQRT2 * V2(t, 1).im;
        B(l + 2 * P1) = SQRT2 * V2(t, M2 + 1).re;
        B(l + 3 * P1) = SQRT2 * V2(t, M2 + 1).im;
    }
    index = index + 4 * P1;
    int l = index;
    for (int j = 2; j <= M2; j++) {
        for (int i = 2; i <= M1; i++) {
            l = l + 1;
            B(l) = SQRT2 * V2(i, j).re;
            B(l + PP) = SQRT2 * V2(i, j).im;
            B(l + 2 * PP) = SQRT2 * V2(i, j + M2).re;
            B(l + 3 * PP) = SQRT2 * V2(i, j + M2).im;
        }
    }
#undef V2
}

/* src/mapping_cpu.jl:59-186 */
void orc_loops_dft_to_beta_3d(double *beta, const double *v, int N1, int N2, int N3, int ld1) {
    int M1 = N1 / 2, M2 = N2 / 2, M3 = N3 / 2;
    int P1 = M1 - 1, P2 = M2 - 1, P3 = M3 - 1;
    int64_t P23 = (int64_t)P2 * P3, P13 = (int64_t)P1 * P3, P12 = (int64_t)P1 * P2, P123 = (int64_t)P1 * P2 * P3;
    const double ms2 = -SQRT2;
#define V3(i, j, k) getc(v, VIDX3(i, j, k))
    B(1) = V3(1, 1, 1).re;
    B(2) = V3(1, 1, M3 + 1).re;
    B(3) = V3(1, M2 + 1, 1).re;
    B(4) = V3(1, M2 + 1, M3 + 1).re;
    B(5) = V3(M1 + 1, 1, 1).re;
    B(6) = V3(M1 + 1, 1, M3 + 1).re;
    B(7) = V3(M1 + 1, M2 + 1, 1).re;
    B(8) = V3(M1 + 1, M2 + 1, M3 + 1).re;
    int64_t index = 8;
    for (int64_t l = index + 1; l <= index + P3; l++) {
        int t = (int)(l - index + 1);
        B(l) = SQRT2 * V3(1, 1, t).re;
        B(l + P3) = SQRT2 * V3(1, 1, t).im;
        B(l + 2 * P3) = SQRT2 * V3(1, M2 + 1, t).re;
        B(l + 3 * P3) = SQRT2 * V3(1, M2 + 1, t).im;
        B(l + 4 * P3) = SQRT2 * V3(M1 + 1, 1, t).re;
        B(l + 5 * P3) = SQRT2 * V3(M1 + 1, 1, t).im;
        B(l + 6 * P3) = SQRT2 * V3(M1 + 1, M2 + 1, t).re;
        B(l + 7 * P3) = SQRT2 * V3(M1 + 1, M2 + 1, t).im;
    }
    index = index + 8 * P3;
    for (int64_t l = index + 1; l <= index + P2; l++) {
        int t = (int)(l - index + 1);
        B(l) = SQRT2 * V3(1, t, 1).re;
        B(l + P2) = SQRT2 * V3(1, t, 1).im;
        B(l + 2 * P2) = SQRT2 * V3(1, t, M3 + 1).re;
        B(l + 3 * P2) = SQRT2 * V3(1, t, M3 + 1).im;
        B(l + 4 * P2) = SQRT2 * V3(M1 + 1, t, 1).re;
        B(l + 5 * P2) = SQRT2 * V3(M1 + 1, t, 1).im;
        B(l + 6 * P2) = SQRT2 * V3(M1 + 1, t, M3 + 1).re;
        B(l + 7 * P2) = SQRT2 * V3(M1 + 1, t, M3 + 1).im;
    }
    index = index + 8 * P2;
    for (int64_t l = index + 1; l <= index + P1; l++) {
        int t = (int)(l - index + 1);
        B(l) = SQRT2 * V3(t, 1, 1).re;
        B(l + P1) = SQRT2 * V3(t, 1, 1).im;
        B(l + 2 * P1) = SQRT2 * V3(t, 1, M3 + 1).re;
        B(l + 3 * P1) = SQRT2 * V3(t, 1, M3 + 1).im;
        B(l + 4 * P1) = SQRT2 * V3(t, M2 + 1, 1).re;
        B(l + 5 * P1) = SQRT2 * V3(t, M2 + 1, 1).im;
        B(l + 6 * P1) = SQRT2 * V3(t, M2 + 1, M3 + 1).re;
        B(l + 7 * P1) = SQRT2 * V3(t, M2 + 1, M3 + 1).im;
    }
    index = index + 8 * P1;
    int64_t l = index;
    for (int k = 2; k <= M3; k++)
        for (int j = 2; j <= M2; j++) {
            l = l + 1;
            B(l) = SQRT2 * V3(1, j, k).re;
            B(l + P23) = SQRT2 * V3(1, j, k).im;
            B(l + 2 * P23) = SQRT2 * V3(1, j + M2, k).re;
            B(l + 3 * P23) = SQRT2 * V3(1, j + M2, k).im;
            B(l + 4 * P23) = SQRT2 * V3(M1 + 1, j, k).re;
            B(l + 5 * P23) = SQRT2 * V3(M1 + 1, j, k).im;
            B(l + 6 * P23) = SQRT2 * V3(M1 + 1, j + M2, k).re;
            B(l + 7 * P23) = SQRT2 * V3(M1 + 1, j + M2, k).im;
        }
    index = index + 8 * P23;
    l = index;
    for (int k = 2; k <= M3; k++)
        for (int i = 2; i <= M1; i++) {
            l = l + 1;
            B(l) = SQRT2 * V3(i, 1, k).re;
            B(l + P13) = SQRT2 * V3(i, 1, k).im;
            B(l + 2 * P13) = SQRT2 * V3(N1 - i - M1 + 2, 1, N3 - k + 2).re;
            B(l + 3 * P13) = ms2 * V3(N1 - i - M1 + 2, 1, N3 - k + 2).im;
            B(l + 4 * P13) = SQRT2 * V3(i, M2 + 1, k).re;
            B(l + 5 * P13) = SQRT2 * V3(i, M2 + 1, k).im;
            B(l + 6 * P13) = SQRT2 * V3(N1 - i - M1 + 2, M2 + 1, N3 - k + 2).re;
            B(l + 7 * P13) = ms2 * V3(N1 - i - M1 + 2, M2 + 1, N3 - k + 2).im;
        }
    index = index + 8 * P13;
    l = index;
    for (int j = 2; j <= M2; j++)
        for (int i = 2; i <= M1; i++) {
            l = l + 1;
            B(l) = SQRT2 * V3(i, j, 1).re;
            B(l + P12) = SQRT2 * V3(i, j, 1).im;
            B(l + 2 * P12) = SQRT2 * V3(N1 - i - M1 + 2, N2 - j + 2, 1).re;
            B(l + 3 * P12) = ms2 * V3(N1 - i - M1 + 2, N2 - j + 2, 1).im;
            B(l + 4 * P12) = SQRT2 * V3(i, j, M3 + 1).re;
            B(l + 5 * P12) = SQRT2 * V3(i, j, M3 + 1).im;
            B(l + 6 * P12) = SQRT2 * V3(N1 - i - M1 + 2, N2 - j + 2, M3 + 1).re;
            B(l + 7 * P12) = ms2 * V3(N1 - i - M1 + 2, N2 - j + 2, M3 + 1).im;
        }
    index = index + 8 * P12;
    l = index;
    for (int k = 2; k <= M3; k++)
        for (int j = 2; j <= M2; j++)
            for (int i = 2; i <= M1; i++) {
                l = l + 1;
                B(l) = SQRT2 * V3(i, j, k).re;
                B(l + P123) = SQRT2 * V3(i, j, k).im;
                B(l + 2 * P123) = SQRT2 * V3(N1 - i - M1 + 2, N2 - j + 2, N3 - k + 2).re;
                B(l + 3 * P123) = ms2 * V3(N1 - i - M1 + 2, N2 - j + 2, N3 - k + 2).im;
                B(l + 4 * P123) = SQRT2 * V3(i, j + M2, k).re;
                B(l + 5 * P123) = SQRT2 * V3(i, j + M2, k).im;
                B(l + 6 * P123) = SQRT2 * V3(N1 - i - M1 + 2, N2 - j - M2 + 2, N3 - k + 2).re;
                B(l + 7 * P123) = ms2 * V3(N1 - i - M1 + 2, N2 - j - M2 + 2, N3 - k + 2).im;
            }
#undef V3
}

/* ======================================================================== */
/*  src/mapping_cpu.jl : beta_to_DFT_{1,2,3}d!  (lines 189-497)              */
/* ======================================================================== */

#define PLUS(r, c)  jl_div_sqrt2(jl_plus_im(B(r), B(c)))   /* (beta[r] + im*beta[c]) / sqrt(2) */
#define MINUS(r, c) jl_div_sqrt2(jl_minus_im(B(r), B(c)))  /* (beta[r] - im*beta[c]) / sqrt(2) */

/* src/mapping_cpu.jl:189-204 */
void orc_loops_beta_to_dft_1d(double *v, const double *beta, int N, int rdft) {
    int M = N / 2;
    setc(v, VIDX1(1), jl_real(B(1)));
    setc(v, VIDX1(M + 1), jl_real(B(2)));
    for (int i = 2; i <= M; i++) setc(v, VIDX1(i), PLUS(i + 1, M + i));
    if (!rdft)
        for (int i = 2; i <= M; i++) setc(v, VIDX1(N - i + 2), MINUS(i + 1, M + i));
}

/* src/mapping_cpu.jl:206-256 */
void orc_loops_beta_to_dft_2d(double *v, const double *beta, int N1, int N2, int rdft) {
    int M1 = N1 / 2, M2 = N2 / 2, P1 = M1 - 1, P2 = M2 - 1;
    int ld1 = rdft ? M1 + 1 : N1;
#define S2(i, j, z) setc(v, VIDX2(i, j), z)
#define G2(i, j) getc(v, VIDX2(i, j))
    S2(1, 1, jl_real(B(1)));
    S2(1, M2 + 1, jl_real(B(2)));
    S2(M1 + 1, 1, jl_real(B(3)));
    S2(M1 + 1, M2 + 1, jl_real(B(4)));
    for (int i = 1; i <= P1; i++) {
        S2(i + 1, 1, PLUS(4 + 4 * P2 + i, 4 + 4 * P2 + P1 + i));
        S2(i + 1, M2 + 1, PLUS(4 + 4 * P2 + 2 * P1 + i, 4 + 4 * P2 + 3 * P1 + i));
    }
    for (int i = 1; i <= P2; i++) {
        S2(1, i + 1, PLUS(4 + i, 4 + P2 + i));
        S2(M1 + 1, i + 1, PLUS(4 + 2 * P2 + i, 4 + 3 * P2 + i));
    }
    int j = 0, c = 0;
    for (int col = 2; col <= M2; col++)
        for (int row = 2; row <= M1; row++) {
            j = j + 1;
            S2(row, col, PLUS(4 + 4 * P2 + 4 * P1 + j, 4 + 4 * P2 + 4 * P1 + P1 * P2 + j));
            S2(M1 - row + 2, N2 - col + 2, PLUS(4 + 4 * P2 + 4 * P1 + 3 * P1 * P2 - c, N1 * N2 - c));
            c = c + 1;
        }
    for (int i = 1; i <= P2; i++) {
        S2(1, M2 + 1 + i, jl_conj(G2(1, M2 - i + 1)));
        S2(M1 + 1, M2 + 1 + i, jl_conj(G2(M1 + 1, M2 - i + 1)));
    }
    if (!rdft) {
        for (int i = 1; i <= P1; i++) {
            S2(N1 - i + 1, 1, MINUS(4 + 4 * P2 + i, 4 + 4 * P2 + P1 + i));
            S2(N1 - i + 1, M2 + 1, MINUS(4 + 4 * P2 + 2 * P1 + i, 4 + 4 * P2 + 3 * P1 + i));
            for (int jj = 1; jj <= P2; jj++) {
                S2(N1 - i + 1, M2 - jj + 1, jl_conj(G2(i + 1, M2 + jj + 1)));
                S2(M1 + i + 1, M2 + jj + 1, jl_conj(G2(M1 - i + 1, M2 - jj + 1)));
            }
        }
    }
#undef S2
#undef G2
}

/* src/mapping_cpu.jl:258-497 */
void orc_loops_beta_to_dft_3d(double *v, const double *beta, int N1, int N2, int N3, int rdft) {
    int M1 = N1 / 2, M2 = N2 / 2, M3 = N3 / 2;
    int64_t P1 = M1 - 1, P2 = M2 - 1, P3 = M3 - 1;
    int ld1 = rdft ? M1 + 1 : N1;
#define S3(i, j, k, z) setc(v, VIDX3(i, j, k), z)
#define G3(i, j, k) getc(v, VIDX3(i, j, k))
    const int64_t E = 8 + 8 * P3 + 8 * P2;                 /* start of the i-edges */
    const int64_t F = 8 + 8 * P3 + 8 * P2 + 8 * P1;        /* start of the faces   */
    S3(1, 1, 1, jl_real(B(1)));
    S3(1, 1, M3 + 1, jl_real(B(2)));
    S3(1, M2 + 1, 1, jl_real(B(3)));
    S3(1, M2 + 1, M3 + 1, jl_real(B(4)));
    S3(M1 + 1, 1, 1, jl_real(B(5)));
    S3(M1 + 1, 1, M3 + 1, jl_real(B(6)));
    S3(M1 + 1, M2 + 1, 1, jl_real(B(7)));
    S3(M1 + 1, M2 + 1, M3 + 1, jl_real(B(8)));

    for (int64_t i = 1; i <= P1; i++) {
        S3(i + 1, 1, 1, PLUS(E + i, E + P1 + i));
        S3(i + 1, 1, M3 + 1, PLUS(E + 2 * P1 + i, E + 3 * P1 + i));
        S3(i + 1, M2 + 1, 1, PLUS(E + 4 * P1 + i, E + 5 * P1 + i));
        S3(i + 1, M2 + 1, M3 + 1, PLUS(E + 6 * P1 + i, E + 7 * P1 + i));
    }
    for (int64_t j = 1; j <= P2; j++) {
        int64_t o = 8 + 8 * P3;
        S3(1, j + 1, 1, PLUS(o + j, o + P2 + j));
        S3(1, j + 1, M3 + 1, PLUS(o + 2 * P2 + j, o + 3 * P2 + j));
        S3(M1 + 1, j + 1, 1, PLUS(o + 4 * P2 + j, o + 5 * P2 + j));
        S3(M1 + 1, j + 1, M3 + 1, PLUS(o + 6 * P2 + j, o + 7 * P2 + j));
    }
    for (int64_t k = 1; k <= P3; k++) {
        S3(1, 1, k + 1, PLUS(8 + k, 8 + P3 + k));
        S3(1, M2 + 1, k + 1, PLUS(8 + 2 * P3 + k, 8 + 3 * P3 + k));
        S3(M1 + 1, 1, k + 1, PLUS(8 + 4 * P3 + k, 8 + 5 * P3 + k));
        S3(M1 + 1, M2 + 1, k + 1, PLUS(8 + 6 * P3 + k, 8 + 7 * P3 + k));
    }
    {   /* faces k in {1, M3+1}: src/mapping_cpu.jl:336-355 */
        int64_t o = F + 8 * P2 * P3 + 8 * P1 * P3;
        for (int64_t j = 1; j <= P2; j++)
            for (int64_t i = 1; i <= P1; i++) {
                int64_t ij = (j - 1) * P1 + i;
                S3(i + 1, j + 1, 1, PLUS(o + ij, o + P1 * P2 + ij));
                S3(M1 - i + 1, N2 - j + 1, 1, MINUS(o + 2 * P1 * P2 + ij, o + 3 * P1 * P2 + ij));
                S3(i + 1, j + 1, M3 + 1, PLUS(o + 4 * P1 * P2 + ij, o + 5 * P1 * P2 + ij));
                S3(M1 - i + 1, N2 - j + 1, M3 + 1, MINUS(o + 6 * P1 * P2 + ij, o + 7 * P1 * P2 + ij));
            }
    }
    {   /* faces j in {1, M2+1}: src/mapping_cpu.jl:357-377 */
        int64_t o = F + 8 * P2 * P3;
        for (int64_t k = 1; k <= P3; k++)
            for (int64_t i = 1; i <= P1; i++) {
                int64_t ik = (k - 1) * P1 + i;
                S3(i + 1, 1, k + 1, PLUS(o + ik, o + P1 * P3 + ik));
                S3(M1 - i + 1, 1, N3 - k + 1, MINUS(o + 2 * P1 * P3 + ik, o + 3 * P1 * P3 + ik));
                S3(i + 1, M2 + 1, k + 1, PLUS(o + 4 * P1 * P3 + ik, o + 5 * P1 * P3 + ik));
                S3(M1 - i + 1, M2 + 1, N3 - k + 1, MINUS(o + 6 * P1 * P3 + ik, o + 7 * P1 * P3 + ik));
            }
    }
    {   /* faces i in {1, M1+1}: src/mapping_cpu.jl:379-399 */
        int64_t o = F;
        for (int64_t k = 1; k <= P3; k++)
            for (int64_t j = 1; j <= P2; j++) {
                int64_t jk = (k - 1) * P2 + j;
                S3(1, j + 1, k + 1, PLUS(o + jk, o + P2 * P3 + jk));
                S3(1, M2 + j + 1, k + 1, PLUS(o + 2 * P2 * P3 + jk, o + 3 * P2 * P3 + jk));
                S3(M1 + 1, j + 1, k + 1, PLUS(o + 4 * P2 * P3 + jk, o + 5 * P2 * P3 + jk));
                S3(M1 + 1, M2 + j + 1, k + 1, PLUS(o + 6 * P2 * P3 + jk, o + 7 * P2 * P3 + jk));
            }
    }
    /* conj mirrors in the planes i in {1, M1+1}: src/mapping_cpu.jl:401-422 */
    for (int64_t j = 1; j <= P2; j++) {
        S3(1, M2 + j + 1, 1, jl_conj(G3(1, M2 - j + 1, 1)));
        S3(M1 + 1, M2 + j + 1, 1, jl_conj(G3(M1 + 1, M2 - j + 1, 1)));
        S3(1, M2 + j + 1, M3 + 1, jl_conj(G3(1, M2 - j + 1, M3 + 1)));
        S3(M1 + 1, M2 + j + 1, M3 + 1, jl_conj(G3(M1 + 1, M2 - j + 1, M3 + 1)));
    }
    for (int64_t k = 1; k <= P3; k++) {
        S3(1, 1, M3 + 1 + k, jl_conj(G3(1, 1, M3 - k + 1)));
        S3(M1 + 1, 1, M3 + 1 + k, jl_conj(G3(M1 + 1, 1, M3 - k + 1)));
        S3(1, M2 + 1, M3 + k + 1, jl_conj(G3(1, M2 + 1, M3 - k + 1)));
        S3(M1 + 1, M2 + 1, M3 + k + 1, jl_conj(G3(M1 + 1, M2 + 1, M3 - k + 1)));
    }
    for (int64_t k = 1; k <= P3; k++)
        for (int64_t j = 1; j <= P2; j++) {
            S3(1, j + 1, M3 + k + 1, jl_conj(G3(1, N2 - j + 1, M3 - k + 1)));
            S3(1, M2 + j + 1, M3 + k + 1, jl_conj(G3(1, M2 - j + 1, M3 - k + 1)));
            S3(M1 + 1, j + 1, M3 + k + 1, jl_conj(G3(M1 + 1, N2 - j + 1, M3 - k + 1)));
            S3(M1 + 1, M2 + j + 1, M3 + k + 1, jl_conj(G3(M1 + 1, M2 - j + 1, M3 - k + 1)));
        }
    {   /* interior: src/mapping_cpu.jl:424-446 */
        int64_t o = F + 8 * P2 * P3 + 8 * P1 * P3 + 8 * P1 * P2;
        int64_t Q = P1 * P2 * P3;
        for (int64_t k = 1; k <= P3; k++)
            for (int64_t j = 1; j <= P2; j++)
                for (int64_t i = 1; i <= P1; i++) {
                    int64_t ijk = (k - 1) * P2 * P1 + (j - 1) * P1 + i;
                    S3(i + 1, j + 1, k + 1, PLUS(o + ijk, o + Q + ijk));
                    S3(M1 - i + 1, N2 - j + 1, N3 - k + 1, MINUS(o + 2 * Q + ijk, o + 3 * Q + ijk));
                    S3(i + 1, M2 + j + 1, k + 1, PLUS(o + 4 * Q + ijk, o + 5 * Q + ijk));
                    S3(M1 - i + 1, M2 - j + 1, N3 - k + 1, MINUS(o + 6 * Q + ijk, o + 7 * Q + ijk));
                }
    }
    if (!rdft) {   /* src/mapping_cpu.jl:448-495 */
        for (int64_t i = 1; i <= P1; i++) {
            S3(M1 + 1 + i, 1, 1, MINUS(E + P1 - i + 1, E + 2 * P1 - i + 1));
            S3(M1 + i + 1, 1, M3 + 1, MINUS(E + 3 * P1 - i + 1, E + 4 * P1 - i + 1));
            S3(M1 + i + 1, M2 + 1, 1, MINUS(E + 5 * P1 - i + 1, E + 6 * P1 - i + 1));
            S3(M1 + i + 1, M2 + 1, M3 + 1, MINUS(E + 7 * P1 - i + 1, E + 8 * P1 - i + 1));
        }
        for (int64_t j = 1; j <= P2; j++)
            for (int64_t i = 1; i <= P1; i++) {
                S3(N1 - i + 1, M2 - j + 1, 1, jl_conj(G3(i + 1, M2 + j + 1, 1)));
                S3(M1 + i + 1, M2 + j + 1, 1, jl_conj(G3(M1 - i + 1, M2 - j + 1, 1)));
                S3(N1 - i + 1, M2 - j + 1, M3 + 1, jl_conj(G3(i + 1, M2 + j + 1, M3 + 1)));
                S3(M1 + i + 1, M2 + j + 1, M3 + 1, jl_conj(G3(M1 - i + 1, M2 - j + 1, M3 + 1)));
            }
        for (int64_t k = 1; k <= P3; k++)
            for (int64_t i = 1; i <= P1; i++) {
                S3(N1 - i + 1, 1, M3 - k + 1, jl_conj(G3(i + 1, 1, M3 + 1 + k)));
                S3(N1 - i + 1, M2 + 1, M3 - k + 1, jl_conj(G3(i + 1, M2 + 1, M3 + k + 1)));
                S3(M1 + i + 1, 1, M3 + k + 1, jl_conj(G3(M1 - i + 1, 1, M3 - k + 1)));
                S3(M1 + i + 1, M2 + 1, M3 + k + 1, jl_conj(G3(M1 - i + 1, M2 + 1, M3 - k + 1)));
            }
        for (int64_t k = 1; k <= P3; k++)
            for (int64_t j = 1; j <= P2; j++)
                for (int64_t i = 1; i <= P1; i++) {
                    S3(M1 + i + 1, M2 + j + 1, M3 + k + 1, jl_conj(G3(M1 - i + 1, M2 - j + 1, M3 - k + 1)));
                    S3(N1 - i + 1, M2 - j + 1, M3 - k + 1, jl_conj(G3(i + 1, M2 + j + 1, M3 + k + 1)));
                    S3(M1 + i + 1, j + 1, M3 + k + 1, jl_conj(G3(M1 - i + 1, N2 - j + 1, M3 - k + 1)));
                    S3(N1 - i + 1, N2 - j + 1, M3 - k + 1, jl_conj(G3(i + 1, j + 1, M3 + k + 1)));
                }
    }
#undef S3
#undef G3
}

/* ======================================================================== */
/*  src/mapping_cpu_kernels.jl : per-index DFT_to_beta  (lines 2-351)        */
/* ======================================================================== */

/* src/mapping_cpu_kernels.jl:11-21 */
static void kern_dft_to_beta_1d(double *beta, const double *v, int N, int M, int64_t i) {
    (void)N;
    if (i == 1) B(i) = getc(v, VIDX1(1)).re;
    else if (i == 2) B(i) = getc(v, VIDX1(M + 1)).re;
    else if (3 <= i && i <= M + 1) B(i) = SQRT2 * getc(v, VIDX1(i - 1)).re;
    else B(i) = SQRT2 * getc(v, VIDX1(i - M)).im;
}

void orc_kern_dft_to_beta_1d(double *beta, const double *v, int N, int ld1) {
    (void)ld1;
    for (int64_t i = 1; i <= N; i++) kern_dft_to_beta_1d(beta, v, N, N / 2, i);
}

/* src/mapping_cpu_kernels.jl:38-87 */
static void kern_dft_to_beta_2d(double *beta, const double *v, int N1, int N2, int ld1, int64_t i) {
    int M1 = N1 / 2, M2 = N2 / 2;
    int64_t P1 = M1 - 1, P2 = M2 - 1, PP = P1 * P2;
    (void)N1;
#define V2(a, b) getc(v, VIDX2(a, b))
    if (i == 1) B(i) = V2(1, 1).re;
    else if (i == 2) B(i) = V2(1, M2 + 1).re;
    else if (i == 3) B(i) = V2(M1 + 1, 1).re;
    else if (i == 4) B(i) = V2(M1 + 1, M2 + 1).re;
    else if (5 <= i && i <= 4 + P2) B(i) = SQRT2 * V2(1, i - 3).re;
    else if (5 + P2 <= i && i <= 4 + 2 * P2) B(i) = SQRT2 * V2(1, i - P2 - 3).im;
    else if (5 + 2 * P2 <= i && i <= 4 + 3 * P2) B(i) = SQRT2 * V2(M1 + 1, i - 2 * P2 - 3).re;
    else if (5 + 3 * P2 <= i && i <= 4 + 4 * P2) B(i) = SQRT2 * V2(M1 + 1, i - 3 * P2 - 3).im;
    else if (5 + 4 * P2 <= i && i <= 4 + 4 * P2 + P1) B(i) = SQRT2 * V2(i - 4 * P2 - 3, 1).re;
    else if (5 + 4 * P2 + P1 <= i && i <= 4 + 4 * P2 + 2 * P1) B(i) = SQRT2 * V2(i - 4 * P2 - P1 - 3, 1).im;
    else if (5 + 4 * P2 + 2 * P1 <= i && i <= 4 + 4 * P2 + 3 * P1) B(i) = SQRT2 * V2(i - 4 * P2 - 2 * P1 - 3, M2 + 1).re;
    else if (5 + 4 * P2 + 3 * P1 <= i && i <= 4 + 4 * P2 + 4 * P1) B(i) = SQRT2 * V2(i - 4 * P2 - 3 * P1 - 3, M2 + 1).im;
    else {
        int64_t base = 4 + 4 * P2 + 4 * P1;
        int64_t blk, j;
        if (i <= base + PP) { blk = 0; j = i - base; }
        else if (i <= base + 2 * PP) { blk = 1; j = i - (base + PP); }
        else if (i <= base + 3 * PP) { blk = 2; j = i - (base + 2 * PP); }
        else { blk = 3; j = i - (base + 3 * PP); }
        int64_t i2 = (j - 1) / P1 + 1;
        int64_t i1 = (j - 1) % P1 + 1;
        if (blk == 0) B(i) = SQRT2 * V2(i1 + 1, i2 + 1).re;
        else if (blk == 1) B(i) = SQRT2 * V2(i1 + 1, i2 + 1).im;
        else if (blk == 2) B(i) = SQRT2 * V2(i1 + 1, i2 + (M2 + 1)).re;
        else B(i) = SQRT2 * V2(i1 + 1, i2 + (M2 + 1)).im;
    }
#undef V2
}

void orc_kern_dft_to_beta_2d(double *beta, const double *v, int N1, int N2, int ld1) {
    for (int64_t i = 1; i <= (int64_t)N1 * N2; i++) kern_dft_to_beta_2d(beta, v, N1, N2, ld1, i);
}

/* src/mapping_cpu_kernels.jl:109-351 */
static void kern_dft_to_beta_3d(double *beta, const double *v, int N1, int N2, int N3, int ld1, int64_t i) {
    int M1 = N1 / 2, M2 = N2 / 2, M3 = N3 / 2;
    int64_t P1 = M1 - 1, P2 = M2 - 1, P3 = M3 - 1;
    int64_t P23 = P2 * P3, P13 = P1 * P3, P12 = P1 * P2, P123 = P1 * P2 * P3;
    const double ms2 = -SQRT2;
#define V3(a, b, c) getc(v, VIDX3(a, b, c))
    if (i == 1) { B(i) = V3(1, 1, 1).re; return; }
    if (i == 2) { B(i) = V3(1, 1, M3 + 1).re; return; }
    if (i == 3) { B(i) = V3(1, M2 + 1, 1).re; return; }
    if (i == 4) { B(i) = V3(1, M2 + 1, M3 + 1).re; return; }
    if (i == 5) { B(i) = V3(M1 + 1, 1, 1).re; return; }
    if (i == 6) { B(i) = V3(M1 + 1, 1, M3 + 1).re; return; }
    if (i == 7) { B(i) = V3(M1 + 1, M2 + 1, 1).re; return; }
    if (i == 8) { B(i) = V3(M1 + 1, M2 + 1, M3 + 1).re; return; }
    /* k-edges, lines 126-141: block b of 8, each P3 long */
    if (i <= 8 + 8 * P3) {
        int64_t b = (i - 9) / P3, t = i - 8 - b * P3;      /* t in 1..P3 */
        int ia = (b / 4) ? M1 + 1 : 1, ja = ((b / 2) % 2) ? M2 + 1 : 1;
        cplx z = V3(ia, ja, t + 1);
        B(i) = SQRT2 * ((b % 2) ? z.im : z.re);
        return;
    }
    /* j-edges, lines 142-157 */
    if (i <= 8 + 8 * P3 + 8 * P2) {
        int64_t r = i - (8 + 8 * P3);
        int64_t b = (r - 1) / P2, t = r - b * P2;
        int ia = (b / 4) ? M1 + 1 : 1, ka = ((b / 2) % 2) ? M3 + 1 : 1;
        cplx z = V3(ia, t + 1, ka);
        B(i) = SQRT2 * ((b % 2) ? z.im : z.re);
        return;
    }
    /* i-edges, lines 158-173 */
    if (i <= 8 + 8 * P3 + 8 * P2 + 8 * P1) {
        int64_t r = i - (8 + 8 * P3 + 8 * P2);
        int64_t b = (r - 1) / P1, t = r - b * P1;
        int ja = (b / 4) ? M2 + 1 : 1, ka = ((b / 2) % 2) ? M3 + 1 : 1;
        cplx z = V3(t + 1, ja, ka);
        B(i) = SQRT2 * ((b % 2) ? z.im : z.re);
        return;
    }
    int64_t F = 8 + 8 * P3 + 8 * P2 + 8 * P1;
    /* faces i, lines 174-213 */
    if (i <= F + 8 * P23) {
        int64_t r = i - F, b = (r - 1) / P23, j = r - b * P23;
        int64_t i3 = (j - 1) / P2 + 1, i2 = (j - 1) % P2 + 1;
        int ia = (b / 4) ? M1 + 1 : 1;
        int64_t jj = ((b / 2) % 2) ? i2 + (M2 + 1) : i2 + 1;
        cplx z = V3(ia, jj, i3 + 1);
        B(i) = SQRT2 * ((b % 2) ? z.im : z.re);
        return;
    }
    /* faces j, lines 214-253 */
    if (i <= F + 8 * P23 + 8 * P13) {
        int64_t r = i - (F + 8 * P23), b = (r - 1) / P13, j = r - b * P13;
        int64_t i3 = (j - 1) / P1 + 1, i1 = (j - 1) % P1 + 1;
        int ja = (b / 4) ? M2 + 1 : 1;
        if (((b / 2) % 2) == 0) {
            cplx z = V3(i1 + 1, ja, i3 + 1);
            B(i) = SQRT2 * ((b % 2) ? z.im : z.re);
        } else {
            cplx z = V3(M1 + 1 - i1, ja, N3 + 1 - i3);
            B(i) = (b % 2) ? ms2 * z.im : SQRT2 * z.re;
        }
        return;
    }
    /* faces k, lines 254-293 */
    if (i <= F + 8 * P23 + 8 * P13 + 8 * P12) {
        int64_t r = i - (F + 8 * P23 + 8 * P13), b = (r - 1) / P12, j = r - b * P12;
        int64_t i2 = (j - 1) / P1 + 1, i1 = (j - 1) % P1 + 1;
        int ka = (b / 4) ? M3 + 1 : 1;
        if (((b / 2) % 2) == 0) {
            cplx z = V3(i1 + 1, i2 + 1, ka);
            B(i) = SQRT2 * ((b % 2) ? z.im : z.re);
        } else {
            cplx z = V3(M1 + 1 - i1, N2 + 1 - i2, ka);
            B(i) = (b % 2) ? ms2 * z.im : SQRT2 * z.re;
        }
        return;
    }
    /* interior, lines 294-350 */
    {
        int64_t r = i - (F + 8 * P23 + 8 * P13 + 8 * P12), b = (r - 1) / P123, j = r - b * P123;
        int64_t i3 = (j - 1) / P12 + 1, kk = (j - 1) % P12 + 1;
        int64_t i2 = (kk - 1) / P1 + 1, i1 = (kk - 1) % P1 + 1;
        cplx z;
        switch (b / 2) {
            case 0: z = V3(i1 + 1, i2 + 1, i3 + 1); break;
            case 1: z = V3(M1 + 1 - i1, N2 + 1 - i2, N3 + 1 - i3); break;
            case 2: z = V3(i1 + 1, i2 + (M2 + 1), i3 + 1); break;
            default: z = V3(M1 + 1 - i1, M2 + 1 - i2, N3 + 1 - i3); break;
        }
        int neg = ((b / 2) == 1 || (b / 2) == 3);
        if (b % 2) B(i) = neg ? ms2 * z.im : SQRT2 * z.im;
        else B(i) = SQRT2 * z.re;
    }
#undef V3
}

void orc_kern_dft_to_beta_3d(double *beta, const double *v, int N1, int N2, int N3, int ld1) {
    int64_t n = (int64_t)N1 * N2 * N3;
    for (int64_t i = 1; i <= n; i++) kern_dft_to_beta_3d(beta, v, N1, N2, N3, ld1, i);
}

/* ======================================================================== */
/*  src/mapping_cpu_kernels.jl : per-index beta_to_DFT  (lines 354-738)      */
/* ======================================================================== */

/* src/mapping_cpu_kernels.jl:363-373 */
void orc_kern_beta_to_dft_1d(double *v, const double *beta, int N, int rdft) {
    int M = N / 2;
    int n = rdft ? M + 1 : N;
    for (int i = 1; i <= n; i++) {
        cplx z;
        if (i == 1) z = jl_real(B(1));
        else if (i == M + 1) z = jl_real(B(2));
        else if (2 <= i && i <= M) z = PLUS(i + 1, M + i);
        else z = MINUS(N + 3 - i, (N + M + 2) - i);
        setc(v, VIDX1(i), z);
    }
}

/* src/mapping_cpu_kernels.jl:392-467 (every branch that fires writes v[i,j]) */
static void kern_beta_to_dft_2d(double *v, const double *beta, int N1, int N2, int ld1, int i, int j) {
    int M1 = N1 / 2, M2 = N2 / 2;
    int64_t P1 = M1 - 1, P2 = M2 - 1, PP = P1 * P2;
#define W2(z) setc(v, VIDX2(i, j), z)
    if (i == 1) { if (j == 1) W2(jl_real(B(1))); else if (j == M2 + 1) W2(jl_real(B(2))); }
    else if (i == M1 + 1) { if (j == 1) W2(jl_real(B(3))); else if (j == M2 + 1) W2(jl_real(B(4))); }

    if (i == 1) {
        if (2 <= j && j <= M2) { int64_t o = 3; W2(PLUS(j + o, j + o + P2)); }
        else if (M2 + 2 <= j && j <= N2) { int64_t o = N2 + 5; W2(MINUS(o - j, o + P2 - j)); }
    } else if (i == M1 + 1) {
        if (2 <= j && j <= M2) { int64_t o = 3 + 2 * P2; W2(PLUS(j + o, j + o + P2)); }
        else if (M2 + 2 <= j && j <= N2) { int64_t o = N2 + 5 + 2 * P2; W2(MINUS(o - j, o + P2 - j)); }
    }
    if (j == 1) {
        if (2 <= i && i <= M1) { int64_t o = 3 + 4 * P2; W2(PLUS(i + o, i + o + P1)); }
        else if (M1 + 2 <= i && i <= N1) { int64_t o = N1 + 5 + 4 * P2; W2(MINUS(o - i, o + P1 - i)); }
    } else if (j == M2 + 1) {
        if (2 <= i && i <= M1) { int64_t o = 3 + 4 * P2 + 2 * P1; W2(PLUS(i + o, i + o + P1)); }
        else if (M1 + 2 <= i && i <= N1) { int64_t o = N1 + 5 + 4 * P2 + 2 * P1; W2(MINUS(o - i, o + P1 - i)); }
    }
    if (2 <= i && i <= M1) {
        if (2 <= j && j <= M2) {
            int64_t o = 4 + 4 * P2 + 4 * P1, idx = (int64_t)(j - 2) * P1 + (i - 1);
            W2(PLUS(o + idx, o + PP + idx));
        } else if (M2 + 2 <= j && j <= N2) {
            int64_t o = 4 + 4 * P2 + 4 * P1 + 2 * PP, idx = (int64_t)(j - M2 - 2) * P1 + (i - 1);
            W2(PLUS(o + idx, o + PP + idx));
        }
    } else if (M1 + 2 <= i && i <= N1) {
        if (2 <= j && j <= M2) {
            int64_t o = 4 + 4 * P2 + 4 * P1 + 3 * PP, idx = (int64_t)(j - 2) * P1 + (i - M1 - 2);
            W2(MINUS(o - idx, o + PP - idx));
        } else if (M2 + 2 <= j && j <= N2) {
            int64_t o = 4 + 4 * P2 + 4 * P1 + PP, idx = (int64_t)(j - M2 - 2) * P1 + (i - M1 - 2);
            W2(MINUS(o - idx, o + PP - idx));
        }
    }
#undef W2
}

/* src/mapping_cpu_kernels.jl:376-390 */
void orc_kern_beta_to_dft_2d(double *v, const double *beta, int N1, int N2, int rdft) {
    int M1 = N1 / 2, ld1 = rdft ? M1 + 1 : N1;
    for (int i = 1; i <= (rdft ? M1 + 1 : N1); i++)
        for (int j = 1; j <= N2; j++) kern_beta_to_dft_2d(v, beta, N1, N2, ld1, i, j);
}

/* src/mapping_cpu_kernels.jl:494-738 */
static void kern_beta_to_dft_3d(double *v, const double *beta, int N1, int N2, int N3, int ld1,
                                int i, int j, int k) {
    int M1 = N1 / 2, M2 = N2 / 2, M3 = N3 / 2;
    int64_t P1 = M1 - 1, P2 = M2 - 1, P3 = M3 - 1;
    int64_t P23 = P2 * P3, P13 = P1 * P3, P12 = P1 * P2, P123 = P1 * P2 * P3;
#define W3(z) setc(v, VIDX3(i, j, k), z)
    /* vertex, lines 495-524 */
    if (i == 1) {
        if (j == 1) { if (k == 1) W3(jl_real(B(1))); else if (k == M3 + 1) W3(jl_real(B(2))); }
        else if (j == M2 + 1) { if (k == 1) W3(jl_real(B(3))); else if (k == M3 + 1) W3(jl_real(B(4))); }
    } else if (i == M1 + 1) {
        if (j == 1) { if (k == 1) W3(jl_real(B(5))); else if (k == M3 + 1) W3(jl_real(B(6))); }
        else if (j == M2 + 1) { if (k == 1) W3(jl_real(B(7))); else if (k == M3 + 1) W3(jl_real(B(8))); }
    }
    /* k-edges, lines 526-555 */
    if ((i == 1 || i == M1 + 1) && (j == 1 || j == M2 + 1)) {
        int64_t s = 2 * (int64_t)((i == M1 + 1) * 2 + (j == M2 + 1)) * P3;
        if (2 <= k && k <= M3) W3(PLUS(k + 7 + s, k + 7 + s + P3));
        else if (M3 + 2 <= k && k <= N3) W3(MINUS(N3 + 9 + s - k, N3 + 9 + s + P3 - k));
    }
    /* j-edges, lines 557-585 */
    if ((i == 1 || i == M1 + 1) && (k == 1 || k == M3 + 1)) {
        int64_t s = 8 * P3 + 2 * (int64_t)((i == M1 + 1) * 2 + (k == M3 + 1)) * P2;
        if (2 <= j && j <= M2) W3(PLUS(j + 7 + s, j + 7 + s + P2));
        else if (M2 + 2 <= j && j <= N2) W3(MINUS(N2 + 9 + s - j, N2 + 9 + s + P2 - j));
    }
    /* i-edges, lines 587-615 */
    if ((j == 1 || j == M2 + 1) && (k == 1 || k == M3 + 1)) {
        int64_t s = 8 * P3 + 8 * P2 + 2 * (int64_t)((j == M2 + 1) * 2 + (k == M3 + 1)) * P1;
        if (2 <= i && i <= M1) W3(PLUS(i + 7 + s, i + 7 + s + P1));
        else if (M1 + 2 <= i && i <= N1) W3(MINUS(N1 + 9 + s - i, N1 + 9 + s + P1 - i));
    }
    const int64_t F = 8 + 8 * P3 + 8 * P2 + 8 * P1;
    /* faces i, lines 618-646 */
    if (i == 1 || i == M1 + 1) {
        int64_t o = F + ((i == M1 + 1) ? 4 * P23 : 0);
        if (2 <= k && k <= M3) {
            if (2 <= j && j <= M2) { int64_t x = (int64_t)(k - 2) * P2 + (j - 1); W3(PLUS(o + x, o + P23 + x)); }
            else if (M2 + 2 <= j && j <= N2) { int64_t x = (int64_t)(k - 2) * P2 + (j - (M2 + 1)); W3(PLUS(o + 2 * P23 + x, o + 3 * P23 + x)); }
        } else if (M3 + 2 <= k && k <= N3) {
            if (2 <= j && j <= M2) { int64_t x = (int64_t)(N3 - k) * P2 + (M2 + 1 - j); W3(MINUS(o + 2 * P23 + x, o + 3 * P23 + x)); }
            else if (M2 + 2 <= j && j <= N2) { int64_t x = (int64_t)(N3 - k) * P2 + (N2 + 1 - j); W3(MINUS(o + x, o + P23 + x)); }
        }
    }
    /* faces j, lines 648-676 */
    if (j == 1 || j == M2 + 1) {
        int64_t o = F + 8 * P23 + ((j == M2 + 1) ? 4 * P13 : 0);
        if (2 <= k && k <= M3) {
            if (2 <= i && i <= M1) { int64_t x = (int64_t)(k - 2) * P1 + (i - 1); W3(PLUS(o + x, o + P13 + x)); }
            else if (M1 + 2 <= i && i <= N1) { int64_t x = (int64_t)(k - 2) * P1 + (i - (M1 + 1)); W3(PLUS(o + 2 * P13 + x, o + 3 * P13 + x)); }
        } else if (M3 + 2 <= k && k <= N3) {
            if (2 <= i && i <= M1) { int64_t x = (int64_t)(N3 - k) * P1 + (M1 + 1 - i); W3(MINUS(o + 2 * P13 + x, o + 3 * P13 + x)); }
            else if (M1 + 2 <= i && i <= N1) { int64_t x = (int64_t)(N3 - k) * P1 + (N1 + 1 - i); W3(MINUS(o + x, o + P13 + x)); }
        }
    }
    /* faces k, lines 678-706 */
    if (k == 1 || k == M3 + 1) {
        int64_t o = F + 8 * P23 + 8 * P13 + ((k == M3 + 1) ? 4 * P12 : 0);
        if (2 <= j && j <= M2) {
            if (2 <= i && i <= M1) { int64_t x = (int64_t)(j - 2) * P1 + (i - 1); W3(PLUS(o + x, o + P12 + x)); }
            else if (M1 + 2 <= i && i <= N1) { int64_t x = (int64_t)(j - 2) * P1 + (i - (M1 + 1)); W3(PLUS(o + 2 * P12 + x, o + 3 * P12 + x)); }
        } else if (M2 + 2 <= j && j <= N2) {
            if (2 <= i && i <= M1) { int64_t x = (int64_t)(N2 - j) * P1 + (M1 + 1 - i); W3(MINUS(o + 2 * P12 + x, o + 3 * P12 + x)); }
            else if (M1 + 2 <= i && i <= N1) { int64_t x = (int64_t)(N2 - j) * P1 + (N1 + 1 - i); W3(MINUS(o + x, o + P12 + x)); }
        }
    }
    /* center, lines 709-737 */
    {
        int64_t o = F + 8 * P23 + 8 * P13 + 8 * P12;
        int iL = (2 <= i && i <= M1), iU = (M1 + 2 <= i && i <= N1);
        int jL = (2 <= j && j <= M2), jU = (M2 + 2 <= j && j <= N2);
        int kL = (2 <= k && k <= M3), kU = (M3 + 2 <= k && k <= N3);
        if (kL) {
            if (jL) {
                if (iL) { int64_t x = (k - 2) * P12 + (j - 2) * P1 + (i - 1); W3(PLUS(o + x, o + P123 + x)); }
                else if (iU) { int64_t x = (k - 2) * P12 + (j - 2) * P1 + (i - (M1 + 1)); W3(PLUS(o + 2 * P123 + x, o + 3 * P123 + x)); }
            } else if (jU) {
                if (iL) { int64_t x = (k - 2) * P12 + (j - (M2 + 2)) * P1 + (i - 1); W3(PLUS(o + 4 * P123 + x, o + 5 * P123 + x)); }
                else if (iU) { int64_t x = (k - 2) * P12 + (j - (M2 + 2)) * P1 + (i - (M1 + 1)); W3(PLUS(o + 6 * P123 + x, o + 7 * P123 + x)); }
            }
        } else if (kU) {
            if (jL) {
                if (iL) { int64_t x = (N3 - k) * P12 + (M2 - j) * P1 + (M1 + 1 - i); W3(MINUS(o + 6 * P123 + x, o + 7 * P123 + x)); }
                else if (iU) { int64_t x = (N3 - k) * P12 + (M2 - j) * P1 + (N1 + 1 - i); W3(MINUS(o + 4 * P123 + x, o + 5 * P123 + x)); }
            } else if (jU) {
                if (iL) { int64_t x = (N3 - k) * P12 + (N2 - j) * P1 + (M1 + 1 - i); W3(MINUS(o + 2 * P123 + x, o + 3 * P123 + x)); }
                else if (iU) { int64_t x = (N3 - k) * P12 + (N2 - j) * P1 + (N1 + 1 - i); W3(MINUS(o + x, o + P123 + x)); }
            }
        }
    }
#undef W3
}

/* src/mapping_cpu_kernels.jl:470-492 */
void orc_kern_beta_to_dft_3d(double *v, const double *beta, int N1, int N2, int N3, int rdft) {
    int M1 = N1 / 2, ld1 = rdft ? M1 + 1 : N1;
    for (int i = 1; i <= (rdft ? M1 + 1 : N1); i++)
        for (int j = 1; j <= N2; j++)
            for (int k = 1; k <= N3; k++) kern_beta_to_dft_3d(v, beta, N1, N2, N3, ld1, i, j, k);
}

/* Convenience dispatchers (dim 1/2/3), mirroring src/fft_utils.jl:144-153 and :195-204 */
void orc_loops_dft_to_beta(double *beta, const double *v, int dim, const int *n, int ld1) {
    if (dim == 1) orc_loops_dft_to_beta_1d(beta, v, n[0], ld1);
    else if (dim == 2) orc_loops_dft_to_beta_2d(beta, v, n[0], n[1], ld1);
    else orc_loops_dft_to_beta_3d(beta, v, n[0], n[1], n[2], ld1);
}
void orc_kern_dft_to_beta(double *beta, const double *v, int dim, const int *n, int ld1) {
    if (dim == 1) orc_kern_dft_to_beta_1d(beta, v, n[0], ld1);
    else if (dim == 2) orc_kern_dft_to_beta_2d(beta, v, n[0], n[1], ld1);
    else orc_kern_dft_to_beta_3d(beta, v, n[0], n[1], n[2], ld1);
}
void orc_loops_beta_to_dft(double *v, const double *beta, int dim, const int *n, int rdft) {
    if (dim == 1) orc_loops_beta_to_dft_1d(v, beta, n[0], rdft);
    else if (dim == 2) orc_loops_beta_to_dft_2d(v, beta, n[0], n[1], rdft);
    else orc_loops_beta_to_dft_3d(v, beta, n[0], n[1], n[2], rdft);
}
void orc_kern_beta_to_dft(double *v, const double *beta, int dim, const int *n, int rdft) {
    if (dim == 1) orc_kern_beta_to_dft_1d(v, beta, n[0], rdft);
    else if (dim == 2) orc_kern_beta_to_dft_2d(v, beta, n[0], n[1], rdft);
    else orc_kern_beta_to_dft_3d(v, beta, n[0], n[1], n[2], rdft);
}
