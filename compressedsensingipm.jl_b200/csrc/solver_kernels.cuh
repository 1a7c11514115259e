// Elementwise + reduction kernels of the interior-point solve, the fused PCG
// and the MadNLP KKT-plugin products.  Every kernel is a grid-stride loop over
// the N beta-space indices; reductions are deterministic (reduce.cuh).
//
// Formulation (src/fft_model.jl:20-34, 91-101): variables [beta; c], slacks
// s1 = c + beta >= 0, s2 = c - beta >= 0 with multipliers z1, z2 >= 0.
// Newton system condensed exactly as src/fft_kkt.jl does: with
// D1 = z1/s1, D2 = z2/s2, L1 = D1 + D2, L2 = D1 - D2,
//     [A'A + L1, L2; L2, L1] [db; dc] = [fb; fc]
// and dc eliminated:  (A'A + Db) db = fb - L2 fc / L1,  Db = 4 D1 D2 / (D1 + D2),
// preconditioned by 1/(1 + Db) — the Schur complement of the reference's
// block preconditioner (src/fft_kkt.jl:46-85) on the same split.
#pragma once
#include <cuda_runtime.h>
#include <float.h>

#include "operator.cuh"
#include "reduce.cuh"

namespace csipm {

#define CSIPM_GRID_LOOP(i, n) for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (n); i += (long long)gridDim.x * blockDim.x)

constexpr int EW_THREADS = 256;

// A kernel scalar given by value or read from device memory when the kernel
// runs (the interior-point solve keeps its per-iteration Newton tolerance on
// the device, so plain launches and graph replays read the same value).
struct DevScalar {
    double v;
    const double* p;
    __host__ __device__ DevScalar(double x = 0.0, const double* q = nullptr) : v(x), p(q) {}
    __device__ __forceinline__ double get() const { return p ? *p : v; }
};

// ------------------------------------------------------------------ CG scalars
// Device scalar block of one CG solve.  rz is double-buffered by iteration parity.
struct CgScalars {
    double rz[2];
    double pq;
    double thresh;      // stop when sqrt(rz) <= thresh
    double rz0;
    int done;           // 1: converged or broke down (later kernels of the solve return at once)
    int iters;          // iterations completed
    int breakdown;      // 1: p'q <= 0 or non-finite
    int pad;
};

// CG scalars of a start whose r.(Minv r) = rz was reduced by the kernel that
// wrote r and p (thresh = atol + rtol*sqrt(rz)); one thread.
__device__ __forceinline__ void cg_start(CgScalars* sc, double rz, double atol, DevScalar rtol_s) {
    const double rtol = rtol_s.get();
    sc->rz[0] = rz;
    sc->rz[1] = 0.0;
    sc->pq = 0.0;
    sc->rz0 = rz;
    sc->thresh = atol + rtol * sqrt(rz);
    sc->iters = 0;
    sc->breakdown = 0;
    sc->done = (sqrt(rz) <= sc->thresh) ? 1 : 0;
    if (!isfinite(rz)) { sc->done = 1; sc->breakdown = 1; }
}

// r = rhs - q (q = (Q + D) x0 computed by the operator), or r = rhs when x0 == 0;
// z = Minv r ; p = z ; rz = r.z ; thresh = atol + rtol*sqrt(rz)
template <typename TV>
__device__ __forceinline__ void cg_init_kernel_body(long long n, const double* __restrict__ rhs, const TV* __restrict__ q, int has_x0,
                               const TV* __restrict__ Minv, TV* __restrict__ r, TV* __restrict__ p,
                               RedWorkspace ws, CgScalars* sc, double atol, DevScalar rtol_s) {
    double acc[1] = {0.0};
    CSIPM_GRID_LOOP(i, n) {
        double rv = rhs[i];
        if (has_x0) rv -= (double)q[i];
        const double zv = Minv ? (double)Minv[i] * rv : rv;
        r[i] = (TV)rv;
        p[i] = (TV)zv;
        acc[0] += rv * zv;
    }
    if (grid_reduce<1>(acc, ws, 0u, 0u) && threadIdx.x == 0) {
        const double rz = ws.out[0];
        sc->rz[0] = rz;
        sc->rz0 = rz;
        sc->thresh = atol + rtol_s.get() * sqrt(rz);
        sc->iters = 0;
        sc->breakdown = 0;
        sc->done = (sqrt(rz) <= sc->thresh) ? 1 : 0;
        if (!isfinite(rz)) { sc->done = 1; sc->breakdown = 1; }
    }
}
template <typename TV>
static __global__ void cg_init_kernel(long long n, const double* __restrict__ rhs, const TV* __restrict__ q, int has_x0,
                               const TV* __restrict__ Minv, TV* __restrict__ r, TV* __restrict__ p,
                               RedWorkspace ws, CgScalars* sc, double atol, DevScalar rtol_s) {
    cg_init_kernel_body<TV>(n, rhs, q, has_x0, Minv, r, p, ws, sc, atol, rtol_s);
}

// alpha = rz/pq ; x += alpha p ; r -= alpha q ; rz' = r.(Minv r)
template <typename TV, typename TX>
__device__ __forceinline__ void cg_update_kernel_body(long long n, int it, TX* __restrict__ x, TV* __restrict__ r, const TV* __restrict__ p,
                                 const TV* __restrict__ q, const TV* __restrict__ Minv, RedWorkspace ws, CgScalars* sc) {
    if (sc->done) return;
    const double pq = sc->pq;
    const double rz = sc->rz[it & 1];
    // breakdown: every block sees the same p.q and returns before touching
    // x or r, so the iterate stays the last good one
    if (!(pq > 0.0) || !isfinite(pq)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) { sc->breakdown = 1; sc->done = 1; }
        return;
    }
    const double alpha = rz / pq;
    double acc[1] = {0.0};
    auto elem = [&](long long k, double xv, double rv0, double pv, double qv, double mv) {
        x[k] = (TX)(xv + alpha * pv);
        const double rv = rv0 - alpha * qv;
        r[k] = (TV)rv;
        acc[0] += Minv ? rv * mv * rv : rv * rv;
    };
    // two elements per trip with all loads issued first (load latency)
    const long long G = (long long)gridDim.x * blockDim.x;
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    for (; i + G < n; i += 2 * G) {
        const long long j = i + G;
        const double xi = (double)x[i], xj = (double)x[j], ri = (double)r[i], rj = (double)r[j];
        const double pi = (double)p[i], pj = (double)p[j], qi = (double)q[i], qj = (double)q[j];
        const double mi = Minv ? (double)Minv[i] : 1.0, mj = Minv ? (double)Minv[j] : 1.0;
        elem(i, xi, ri, pi, qi, mi);
        elem(j, xj, rj, pj, qj, mj);
    }
    if (i < n) elem(i, (double)x[i], (double)r[i], (double)p[i], (double)q[i], Minv ? (double)Minv[i] : 1.0);
    if (grid_reduce<1>(acc, ws, 0u, 0u) && threadIdx.x == 0) {
        const double rzn = ws.out[0];
        sc->rz[(it + 1) & 1] = rzn;
        sc->iters += 1;     // counted on the device: graph replays reuse the same `it` values
        if (!isfinite(rzn)) { sc->breakdown = 1; sc->done = 1; }
        else if (sqrt(rzn) <= sc->thresh) sc->done = 1;
    }
}
template <typename TV, typename TX>
static __global__ void cg_update_kernel(long long n, int it, TX* __restrict__ x, TV* __restrict__ r, const TV* __restrict__ p,
                                 const TV* __restrict__ q, const TV* __restrict__ Minv, RedWorkspace ws, CgScalars* sc) {
    cg_update_kernel_body<TV, TX>(n, it, x, r, p, q, Minv, ws, sc);
}

// p = Minv r + (rz'/rz) p
template <typename TV>
__device__ __forceinline__ void cg_pupdate_kernel_body(long long n, int it, const TV* __restrict__ r, const TV* __restrict__ Minv, TV* __restrict__ p,
                                  const CgScalars* sc) {
    if (sc->done) return;
    const double b = sc->rz[(it + 1) & 1] / sc->rz[it & 1];
    const long long G = (long long)gridDim.x * blockDim.x;
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    for (; i + G < n; i += 2 * G) {
        const long long j = i + G;
        const double ri = (double)r[i], rj = (double)r[j], pi = (double)p[i], pj = (double)p[j];
        const double mi = Minv ? (double)Minv[i] : 1.0, mj = Minv ? (double)Minv[j] : 1.0;
        p[i] = (TV)(mi * ri + b * pi);
        p[j] = (TV)(mj * rj + b * pj);
    }
    if (i < n) p[i] = (TV)((Minv ? (double)Minv[i] : 1.0) * (double)r[i] + b * (double)p[i]);
}
template <typename TV>
static __global__ void cg_pupdate_kernel(long long n, int it, const TV* __restrict__ r, const TV* __restrict__ Minv, TV* __restrict__ p,
                                  const CgScalars* sc) {
    cg_pupdate_kernel_body<TV>(n, it, r, Minv, p, sc);
}

// Mixed precision: r = rhs - q in FP64 with r.(Minv r) (the refinement residual)
static __global__ void resid64_kernel(long long n, const double* __restrict__ rhs, const double* __restrict__ q,
                                      const double* __restrict__ Minv, double* __restrict__ r, RedWorkspace ws) {
    double acc[1] = {0.0};
    CSIPM_GRID_LOOP(i, n) {
        const double rv = rhs[i] - q[i];
        r[i] = rv;
        acc[0] += Minv ? rv * Minv[i] * rv : rv * rv;
    }
    grid_reduce<1>(acc, ws, 0u, 0u);
}

// x += d (FP32 correction into the FP64 iterate)
static __global__ void add_f32_kernel(long long n, const float* __restrict__ d, double* __restrict__ x) {
    CSIPM_GRID_LOOP(i, n) x[i] += (double)d[i];
}

// ------------------------------------------------------------------ IPM state
// Reductions of the residual kernel (component index):
enum { RR_SZ = 0, RR_BB, RR_BQB, RR_L1, RR_GINF, RR_RDINF, RR_RCINF, RR_SUMC, RR_RZ, RR_N };
constexpr unsigned RR_MAXMASK = (1u << RR_GINF) | (1u << RR_RDINF) | (1u << RR_RCINF);

// beta = soft(b, lambda); reduce max|beta| and max|b|
__device__ __forceinline__ void ipm_init1_kernel_body(long long n, const double* __restrict__ b, double lam, double* __restrict__ beta,
                                 RedWorkspace ws) {
    double acc[2] = {0.0, 0.0};
    CSIPM_GRID_LOOP(i, n) {
        const double bi = b[i];
        const double a = fabs(bi) - lam;
        const double v = a > 0.0 ? copysign(a, bi) : 0.0;
        beta[i] = v;
        acc[0] = fmax(acc[0], fabs(v));
        acc[1] = fmax(acc[1], fabs(bi));
    }
    grid_reduce<2>(acc, ws, 3u, 0u);
}
static __global__ void ipm_init1_kernel(long long n, const double* __restrict__ b, double lam, double* __restrict__ beta,
                                 RedWorkspace ws) {
    ipm_init1_kernel_body(n, b, lam, beta, ws);
}

// Dual start from the clipped gradient with lz = max(lambda, 1e-3 |b|_inf, 1e-12)
// (the floor keeps lambda = 0 interior); c = |beta| + mu0/min(z1,z2),
// mu0 = 0.1*lz*max(1e-3, max|beta|).  mx = {max|beta|, max|b|}.
// The slacks s1 = c + beta, s2 = c - beta are the stored variables from here
// on (MadNLP's slack formulation): recomputing them from c and beta would
// cancel catastrophically once a bound is nearly active.
__device__ __forceinline__ void ipm_init2_kernel_body(long long n, const double* __restrict__ b, const double* __restrict__ Qb, double lam,
                                 const double* __restrict__ beta, const double* __restrict__ mx,
                                 double* __restrict__ s1, double* __restrict__ s2, double* __restrict__ z1,
                                 double* __restrict__ z2) {
    const double lz = fmax(fmax(lam, 1e-3 * mx[1]), 1e-12);
    const double mu0 = 0.1 * lz * fmax(1e-3, mx[0]);
    CSIPM_GRID_LOOP(i, n) {
        double g = Qb[i] - b[i];
        g = fmin(fmax(g, -0.5 * lz), 0.5 * lz);
        const double a = 0.5 * (lz + g), d = 0.5 * (lz - g);
        z1[i] = a;
        z2[i] = d;
        const double be = beta[i];
        const double ce = fabs(be) + mu0 / fmin(a, d);
        s1[i] = ce + be;
        s2[i] = ce - be;
    }
}
static __global__ void ipm_init2_kernel(long long n, const double* __restrict__ b, const double* __restrict__ Qb, double lam,
                                 const double* __restrict__ beta, const double* __restrict__ mx,
                                 double* __restrict__ s1, double* __restrict__ s2, double* __restrict__ z1,
                                 double* __restrict__ z2) {
    ipm_init2_kernel_body(n, b, Qb, lam, beta, mx, s1, s2, z1, z2);
}

// Per-element quantities shared by every direction of one iteration:
// 1/s1, 1/s2, D1 = z1/s1, D2 = z2/s2, L2 = D1 - D2 and 1/L1 with L1 = D1 + D2
// (three divisions; FP64 division is the expensive part of these kernels).
struct ElemPre { double a, d, is1, is2, D1, D2, L2, iL1; };

// One FP64 division per element: with p = s1 s2 and w = a s2 + d s1 (so
// D1 + D2 = w/p), R = 1/(p w) gives 1/s1 = s2 w R, 1/s2 = s1 w R and
// 1/(D1 + D2) = p p R.  Slacks and multipliers are strictly positive inside
// the interior-point loop, so p w > 0; three IEEE divisions per element kept
// the FP64 pipe of the step-statistics pass 41-47% busy.
__device__ __forceinline__ ElemPre elem_pre(double s1, double s2, double a, double d) {
    ElemPre e;
    e.a = a;
    e.d = d;
    const double p = s1 * s2;
    const double w = fma(a, s2, d * s1);
    const double R = 1.0 / (p * w);
    const double u = w * R;   // 1/p
    e.is1 = s2 * u;
    e.is2 = s1 * u;
    e.D1 = a * e.is1;
    e.D2 = d * e.is2;
    e.L2 = e.D1 - e.D2;
    e.iL1 = p * (p * R);
    return e;
}

// Barrier diagonal of the condensed Schur system, its Jacobi preconditioner
// and the fc weight of the right-hand side, from one division: with
// w = a s2 + d s1 and q = 4 a d, Db = 4 D1 D2/(D1 + D2) = q/w,
// Minv = 1/(1 + Db) = w/(w + q) and L2/L1 = (D1 - D2)/(D1 + D2) = (a s2 - d s1)/w,
// all from R = 1/(w (w + q)).  The residual pass and the lazy FP64 diagonal
// kernel both use it, so their Db and Minv agree bit for bit.
struct ElemDiag { double db, mi, l2l1; };

__device__ __forceinline__ ElemDiag elem_diag(double s1, double s2, double a, double d, bool precond) {
    const double as2 = a * s2, ds1 = d * s1;
    const double w = as2 + ds1, q = 4.0 * (a * d);
    ElemDiag g;
    double rw;
    if (precond) {
        const double R = 1.0 / (w * (w + q));
        rw = (w + q) * R;
        g.mi = w * (w * R);
    } else {
        rw = 1.0 / w;
        g.mi = 1.0;
    }
    g.db = q * rw;
    g.l2l1 = (as2 - ds1) * rw;
    return g;
}

// Newton direction of one element given db, the centring target sigmu and the
// second-order correction (cor1, cor2):
//   h1 = (sigmu - s1 z1 - cor1)/s1,  h2 likewise,  fc = -(lambda - z1 - z2) + h1 + h2,
//   dc = (fc - L2 db)/L1,  ds1 = dc + db,  ds2 = dc - db,  dz = h - D ds.
// The affine direction (sigmu = 0, no correction) has h1 = -z1, h2 = -z2.
struct ElemDir { double dc, ds1, ds2, dz1, dz2; };

__device__ __forceinline__ ElemDir elem_dir(const ElemPre& e, double lam, double sigmu, double cor1, double cor2,
                                            double db) {
    const double h1 = (sigmu - cor1) * e.is1 - e.a;
    const double h2 = (sigmu - cor2) * e.is2 - e.d;
    const double fc = -(lam - e.a - e.d) + h1 + h2;
    ElemDir o;
    o.dc = (fc - e.L2 * db) * e.iL1;
    o.ds1 = o.dc + db;
    o.ds2 = o.dc - db;
    o.dz1 = h1 - e.D1 * o.ds1;
    o.dz2 = h2 - e.D2 * o.ds2;
    return o;
}

__device__ __forceinline__ ElemDir elem_affine(const ElemPre& e, double lam, double db) {
    const double fc = -lam;   // -(lambda - z1 - z2) + h1 + h2 with h = -z
    ElemDir o;
    o.dc = (fc - e.L2 * db) * e.iL1;
    o.ds1 = o.dc + db;
    o.ds2 = o.dc - db;
    o.dz1 = -e.a - e.D1 * o.ds1;
    o.dz2 = -e.d - e.D2 * o.ds2;
    return o;
}

// rhs = fb - L2 fc / L1 with fb = -rd + h1 - h2 (corrector: sigmu and the
// second-order correction of the affine direction dba).  With rp (the
// predictor solve's residual rhs_p - K dba) the corrector's warm-start
// residual rhs - K dba = rhs - rhs_p + rp replaces rd (rd is not needed after
// this pass; rhs still holds rhs_p on entry); with x0 the warm start
// x0 = dba is written as well.
//
// With cr (FP32 corrector CG, rp given): the CG starts here instead of rd:
// r = the warm-start residual, p = Minv r (cm: the rounded preconditioner,
// null without one), r.(Minv r) reduced and the CG scalars set.  rp may be
// the same vector as cr (read, then overwritten, by the same thread).
template <typename TR, typename TD>
__device__ __forceinline__ void ipm_rhs_kernel_body(long long n, double lam, const double* __restrict__ s1v, const double* __restrict__ s2v,
                               const double* __restrict__ z1, const double* __restrict__ z2, double* rd,
                               const TD* __restrict__ dba, const double* __restrict__ sigmu_p, double* rhs,
                               const TR* rp, TD* __restrict__ x0, float* cr, float* __restrict__ cp,
                               const float* __restrict__ cm, CgScalars* csc, RedWorkspace ws, DevScalar crtol) {
    const double sigmu = sigmu_p ? *sigmu_p : 0.0;
    double acc[1] = {0.0};
    CSIPM_GRID_LOOP(i, n) {
        const ElemPre e = elem_pre(s1v[i], s2v[i], z1[i], z2[i]);
        double cor1 = 0.0, cor2 = 0.0;
        if (dba) {
            const ElemDir f = elem_affine(e, lam, (double)dba[i]);
            cor1 = f.ds1 * f.dz1;
            cor2 = f.ds2 * f.dz2;
        }
        const double h1 = (sigmu - cor1) * e.is1 - e.a;
        const double h2 = (sigmu - cor2) * e.is2 - e.d;
        const double fb = -rd[i] + h1 - h2;
        const double fc = -(lam - e.a - e.d) + h1 + h2;
        const double rn = fb - e.L2 * fc * e.iL1;
        if (cr) {
            const double r0 = rn - rhs[i] + (double)rp[i];
            const double zv = cm ? (double)cm[i] * r0 : r0;
            cr[i] = (float)r0;
            cp[i] = (float)zv;
            acc[0] += r0 * zv;
        } else if (rp) {
            rd[i] = rn - rhs[i] + (double)rp[i];
        }
        rhs[i] = rn;
        if (x0) x0[i] = dba[i];
    }
    if (cr && grid_reduce<1>(acc, ws, 0u, 0u) && threadIdx.x == 0) cg_start(csc, ws.out[0], 0.0, crtol);
}
template <typename TR, typename TD>
static __global__ void ipm_rhs_kernel(long long n, double lam, const double* __restrict__ s1v, const double* __restrict__ s2v,
                               const double* __restrict__ z1, const double* __restrict__ z2, double* rd,
                               const TD* __restrict__ dba, const double* __restrict__ sigmu_p, double* rhs,
                               const TR* rp, TD* __restrict__ x0, float* cr, float* __restrict__ cp,
                               const float* __restrict__ cm, CgScalars* csc, RedWorkspace ws, DevScalar crtol) {
    ipm_rhs_kernel_body<TR, TD>(n, lam, s1v, s2v, z1, z2, rd, dba, sigmu_p, rhs, rp, x0, cr, cp, cm, csc, ws, crtol);
}

// ------------------------------------------------------------------ IPM control
// Device control block of csipm_solve.  After every residual pass a
// one-thread kernel (ipm_stop_kernel) turns the pass's reductions into mu,
// the LASSO duality gap and the scaled KKT error, decides whether to stop,
// and sets the Newton tolerance of the coming solves (forcing term); the
// other kernels read mu, eta and the tolerances from here.  The host loop
// reads the block once per iteration; a CUDA graph of whole iterations reads
// nothing back until it ends.
enum { IPM_RUNNING = 0, IPM_CONVERGED = 1, IPM_MAXITER = 2, IPM_NONFINITE = 3, IPM_ABORT = 4 };
struct IpmCtl {
    // set by the host at the start of a solve
    double tol, rt_opt, forcing, rt_floor, rin_floor, z0sq, kkt_scale, lam, two_n;
    int max_iter;
    int k;              // iteration whose stop test ran last (-1 before the first)
    // per iteration
    double rt;          // relative tolerance of this iteration's Newton solves
    double rin;         // max(rt, rin_floor): round 0 of a mixed-precision solve
    double rt_next;     // the next iteration's (its residual pass starts the predictor CG)
    double rin_next;
    double mu, gap, kkt, F, obj, dual_inf, eta;
    int status;         // IPM_*
    int cg_iter;        // CG iterations run inside graph replays
    int graph_iters;    // iterations completed inside graph replays
    int abort_cg;       // graph replay stopped by a CG loop: 1 predictor, 2 corrector
    int cg_done_last;   // pad
    int pad;
};

// R: the residual pass's reductions (RR_*).  One thread.  With a conditional
// handle (graph replays) the loop goes on while the status is IPM_RUNNING.
__device__ __forceinline__ void ipm_stop_kernel_body(const double* __restrict__ R, IpmCtl* __restrict__ c, int in_graph,
                                       cudaGraphConditionalHandle hnd) {
    const int k = c->k + 1;
    c->k = k;
    const double mu = R[RR_SZ] / c->two_n;
    const double usq = c->z0sq - 2.0 * R[RR_BB] + R[RR_BQB];
    const double F = 0.5 * usq + c->lam * R[RR_L1];
    const double th = R[RR_GINF] > 0.0 ? fmin(1.0, c->lam / R[RR_GINF]) : 1.0;
    const double D = th * (c->z0sq - R[RR_BB]) - 0.5 * th * th * usq;
    const double gap = (F - D) / fmax(fabs(F), 1e-300);
    // scaled KKT error: the criterion that still applies when lambda = 0
    // makes the LASSO dual bound degenerate
    const double kkt = fmax(fmax(R[RR_RDINF], R[RR_RCINF]) / c->kkt_scale, R[RR_SZ] / fmax(1.0, fabs(F)));
    c->mu = mu;
    c->gap = gap;
    c->kkt = kkt;
    c->F = F;
    c->obj = 0.5 * R[RR_BQB] - R[RR_BB] + c->lam * R[RR_SUMC];
    c->dual_inf = R[RR_RDINF];
    c->eta = fmax(0.99, 1.0 - mu);
    int st = IPM_RUNNING;
    if (!isfinite(mu) || !isfinite(gap)) st = IPM_NONFINITE;
    else if (gap <= c->tol || kkt <= c->tol) st = IPM_CONVERGED;
    else if (k >= c->max_iter) st = IPM_MAXITER;
    c->status = st;
    // this iteration solves at the tolerance its residual pass started with;
    // the next one at the forcing term of this gap
    c->rt = c->rt_next;
    c->rin = c->rin_next;
    const double rn = c->forcing > 0.0 ? fmin(c->rt_opt, fmax(c->rt_floor, c->forcing * gap)) : c->rt_opt;
    c->rt_next = rn;
    c->rin_next = fmax(rn, c->rin_floor);
    if (in_graph) {
        c->graph_iters += 1;
        cudaGraphSetConditional(hnd, st == IPM_RUNNING ? 1u : 0u);
    }
}
static __global__ void ipm_stop_kernel(const double* __restrict__ R, IpmCtl* __restrict__ c, int in_graph,
                                       cudaGraphConditionalHandle hnd) {
    ipm_stop_kernel_body(R, c, in_graph, hnd);
}

// Graph replays: opens a CG loop (a conditional while node) unless its start
// already met the tolerance.  One thread.
static __global__ void cg_arm_kernel(cudaGraphConditionalHandle hnd, const CgScalars* __restrict__ sc) {
    cudaGraphSetConditional(hnd, sc->done ? 0u : 1u);
}

// Graph replays: after a CG loop, count its iterations and let the rest of
// the iteration run only if it converged (a breakdown, or the loop's cap
// below the solve's iteration cap, hands the iteration back to the host).
static __global__ void ipm_cg_check_kernel(const CgScalars* __restrict__ sc, IpmCtl* __restrict__ c, int which,
                                           int cap_is_limit, cudaGraphConditionalHandle if_hnd,
                                           cudaGraphConditionalHandle loop_hnd) {
    const bool ok = !sc->breakdown && (sc->done || cap_is_limit);
    c->cg_iter += sc->iters;
    if (!ok) {
        c->status = IPM_ABORT;
        c->abort_cg = which;
        cudaGraphSetConditional(loop_hnd, 0u);
    }
    cudaGraphSetConditional(if_hnd, ok ? 1u : 0u);
}

// Step statistics of a direction: min ratios (primal, dual) and the sums for mu_aff.
enum { SS_MINP = 0, SS_MIND, SS_SZ, SS_CROSS, SS_DD, SS_N };
constexpr unsigned SS_MINMASK = (1u << SS_MINP) | (1u << SS_MIND);

// Running minimum of v/w (v >= 0, w > 0) kept as a fraction num/den, compared
// by cross-multiplication: one division per thread instead of one per element.
struct MinRatio {
    double num = 1.0, den = 0.0;   // 1/0: +infinity
    __device__ __forceinline__ void add(double v, double w) {
        if (v * den < num * w) { num = v; den = w; }
    }
    __device__ __forceinline__ double value() const { return den > 0.0 ? num / den : DBL_MAX; }
};

// TD: type the Newton directions are stored in (FP32 in loose mixed precision)
template <typename TD>
__device__ __forceinline__ void ipm_stepstats_kernel_body(long long n, double lam, const double* __restrict__ s1v, const double* __restrict__ s2v,
                     const double* __restrict__ z1, const double* __restrict__ z2, const TD* __restrict__ dba,
                     const double* __restrict__ sigmu_p, const TD* __restrict__ db, RedWorkspace ws) {
    const double sigmu = sigmu_p ? *sigmu_p : 0.0;
    double acc[SS_N] = {DBL_MAX, DBL_MAX, 0.0, 0.0, 0.0};
    MinRatio mp, md;
    auto elem = [&](double s1, double s2, double a, double d, double xa, double x) {
        const ElemPre e = elem_pre(s1, s2, a, d);
        ElemDir o;
        if (dba) {
            const ElemDir f = elem_affine(e, lam, xa);
            o = elem_dir(e, lam, sigmu, f.ds1 * f.dz1, f.ds2 * f.dz2, x);
        } else {
            o = elem_affine(e, lam, x);
        }
        if (o.ds1 < 0.0) mp.add(s1, -o.ds1);
        if (o.ds2 < 0.0) mp.add(s2, -o.ds2);
        if (o.dz1 < 0.0) md.add(a, -o.dz1);
        if (o.dz2 < 0.0) md.add(d, -o.dz2);
        acc[SS_SZ] += s1 * a + s2 * d;
        acc[SS_CROSS] += s1 * o.dz1 + o.ds1 * a + s2 * o.dz2 + o.ds2 * d;
        acc[SS_DD] += o.ds1 * o.dz1 + o.ds2 * o.dz2;
    };
    // two elements per trip, all their loads issued before the FP64 math
    // (the kernel is otherwise bound by load latency at its occupancy)
    const long long G = (long long)gridDim.x * blockDim.x;
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    for (; i + G < n; i += 2 * G) {
        const long long j = i + G;
        const double s1i = s1v[i], s1j = s1v[j], s2i = s2v[i], s2j = s2v[j];
        const double ai = z1[i], aj = z1[j], di = z2[i], dj = z2[j];
        const double xai = dba ? (double)dba[i] : 0.0, xaj = dba ? (double)dba[j] : 0.0;
        const double xi = (double)db[i], xj = (double)db[j];
        elem(s1i, s2i, ai, di, xai, xi);
        elem(s1j, s2j, aj, dj, xaj, xj);
    }
    if (i < n) elem(s1v[i], s2v[i], z1[i], z2[i], dba ? (double)dba[i] : 0.0, (double)db[i]);
    acc[SS_MINP] = mp.value();
    acc[SS_MIND] = md.value();
    grid_reduce<SS_N>(acc, ws, 0u, SS_MINMASK);
}
template <typename TD>
static __global__ void __launch_bounds__(EW_THREADS, 3)
ipm_stepstats_kernel(long long n, double lam, const double* __restrict__ s1v, const double* __restrict__ s2v,
                     const double* __restrict__ z1, const double* __restrict__ z2, const TD* __restrict__ dba,
                     const double* __restrict__ sigmu_p, const TD* __restrict__ db, RedWorkspace ws) {
    ipm_stepstats_kernel_body<TD>(n, lam, s1v, s2v, z1, z2, dba, sigmu_p, db, ws);
}

// Centring target after the predictor (Mehrotra): a = min(1, primal and dual
// ratios), mu_aff = (s'z + a cross + a^2 dd)/(2n), sigma = min(1, mu_aff/mu)^3;
// q: the predictor's step statistics.  One thread.
__device__ __forceinline__ void ipm_sigma_kernel_body(const double* __restrict__ q, const IpmCtl* __restrict__ c,
                                        double* __restrict__ sigmu) {
    const double mu = c->mu, two_n = c->two_n;
    const double a = fmin(1.0, fmin(q[SS_MINP], q[SS_MIND]));
    const double mu_aff = (q[SS_SZ] + a * q[SS_CROSS] + a * a * q[SS_DD]) / two_n;
    const double r = fmin(1.0, fmax(mu_aff, 0.0) / mu);   // sigma <= 1: the target never rises above mu
    *sigmu = r * r * r * mu;
}
static __global__ void ipm_sigma_kernel(const double* __restrict__ q, const IpmCtl* __restrict__ c,
                                        double* __restrict__ sigmu) {
    ipm_sigma_kernel_body(q, c, sigmu);
}

// Step length after the corrector: min over primal and dual of
// min(1, eta * ratio) (the same step for both), eta = max(0.99, 1 - mu) from
// the control block.  One thread.
__device__ __forceinline__ void ipm_alpha_kernel_body(const double* __restrict__ q, const IpmCtl* __restrict__ c,
                                        double* __restrict__ alpha) {
    const double eta = c->eta;
    const double ap = fmin(1.0, eta * q[SS_MINP]);
    const double ad = fmin(1.0, eta * q[SS_MIND]);
    *alpha = fmin(ap, ad);
}
static __global__ void ipm_alpha_kernel(const double* __restrict__ q, const IpmCtl* __restrict__ c,
                                        double* __restrict__ alpha) {
    ipm_alpha_kernel_body(q, c, alpha);
}

// ------------------------------------------------------------------ ADMM (src/admm.jl)
// b = A'z0 + rho z - y
static __global__ void admm_rhs_kernel(long long n, const double* __restrict__ bv, const double* __restrict__ z,
                                       const double* __restrict__ y, double rho, double* __restrict__ b) {
    CSIPM_GRID_LOOP(i, n) b[i] = bv[i] + rho * z[i] - y[i];
}

// z1 = soft(x1 + y0/rho, lambda/rho), y1 = y0 + rho (x1 - z1), the squared
// norms of x1 - x0, y1 - y0, z1 - z0, and the next right-hand side
// A'z0 + rho z1 - y1 (z, y updated in place)
static __global__ void admm_update_kernel(long long n, const double* __restrict__ bv, const double* __restrict__ x1,
                                          const double* __restrict__ x0, double* __restrict__ z,
                                          double* __restrict__ y, double rho, double lam, double* __restrict__ b,
                                          RedWorkspace ws) {
    double acc[3] = {0.0, 0.0, 0.0};
    const double thre = lam / rho;
    CSIPM_GRID_LOOP(i, n) {
        const double xv = x1[i], y0 = y[i], z0 = z[i];
        const double v = xv + y0 / rho;
        const double z1 = v > thre ? v - thre : (v < -thre ? v + thre : 0.0);
        const double y1 = y0 + rho * (xv - z1);
        const double dx = xv - x0[i], dy = y1 - y0, dz = z1 - z0;
        acc[0] += dx * dx;
        acc[1] += dy * dy;
        acc[2] += dz * dz;
        z[i] = z1;
        y[i] = y1;
        b[i] = bv[i] + rho * z1 - y1;
    }
    grid_reduce<3>(acc, ws, 0u, 0u);
}

// One pass per interior-point iteration over the state: first the pending
// step of the previous iteration on the slacks and multipliers (beta was
// stepped before the A'A product that produced Qb), when dba/db are given:
// the corrector direction of each element recomputed from the stored
// directions, s += alpha ds, z += alpha dz; then the dual residual
// rd = Qb - b - z1 + z2 and the scalar diagnostics (reductions RR_*), the
// barrier diagonals of the condensed Schur system Db = 4 D1 D2/(D1 + D2),
// Minv = 1/(1 + Db) (FP64 when Db is given, FP32 copies for mixed
// precision), and the predictor right-hand side (h1 = -z1, h2 = -z2,
// fc = -lambda).
template <typename TV, typename TD>
__device__ __forceinline__ void ipm_resdiag_kernel_body(long long n, const double* __restrict__ b, const double* __restrict__ Qb, double lam,
                   const double* __restrict__ beta, double* __restrict__ s1v, double* __restrict__ s2v,
                   double* __restrict__ z1, double* __restrict__ z2, const TD* __restrict__ dba,
                   const TD* __restrict__ db, const double* __restrict__ sigmu_p,
                   const double* __restrict__ alpha_p, double* __restrict__ rd, double* __restrict__ Db,
                   double* __restrict__ Minv, TV* __restrict__ Db_lo, TV* __restrict__ Minv_lo, int precond,
                   double* __restrict__ rhs, RedWorkspace ws, TV* __restrict__ cr, TV* __restrict__ cp,
                   CgScalars* csc, DevScalar crtol) {
    double acc[RR_N] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    const bool step = db != nullptr;
    const double sigmu = step ? *sigmu_p : 0.0;
    const double alpha = step ? *alpha_p : 0.0;
    auto elem = [&](long long i, double s1, double s2, double a, double d, double xa, double x, double be, double q,
                    double bb) {
        if (step) {
            const ElemPre e = elem_pre(s1, s2, a, d);
            const ElemDir f = elem_affine(e, lam, xa);
            const ElemDir o = elem_dir(e, lam, sigmu, f.ds1 * f.dz1, f.ds2 * f.dz2, x);
            s1 += alpha * o.ds1;
            s2 += alpha * o.ds2;
            a += alpha * o.dz1;
            d += alpha * o.dz2;
            s1v[i] = s1;
            s2v[i] = s2;
            z1[i] = a;
            z2[i] = d;
        }
        const double ce = 0.5 * (s1 + s2);
        const double r = q - bb - a + d;
        rd[i] = r;
        const double rc = lam - a - d;
        acc[RR_SZ] += s1 * a + s2 * d;
        acc[RR_BB] += bb * be;
        acc[RR_BQB] += be * q;
        acc[RR_L1] += fabs(be);
        acc[RR_GINF] = fmax(acc[RR_GINF], fabs(bb - q));
        acc[RR_RDINF] = fmax(acc[RR_RDINF], fabs(r));
        acc[RR_RCINF] = fmax(acc[RR_RCINF], fabs(rc));
        acc[RR_SUMC] += ce;
        const ElemDiag g = elem_diag(s1, s2, a, d, precond);
        const double dbv = g.db, mi = g.mi;
        if (Db) { Db[i] = dbv; Minv[i] = mi; }
        if (Db_lo) { Db_lo[i] = (TV)dbv; Minv_lo[i] = (TV)mi; }
        const double v = -r - a + d + lam * g.l2l1;
        rhs[i] = v;
        if (cr) {
            // start of the predictor's FP32 CG (r = rhs, p = Minv r, from x = 0),
            // with the rounded preconditioner the CG kernels read
            const double zv = (double)(TV)mi * v;
            cr[i] = (TV)v;
            cp[i] = (TV)zv;
            acc[RR_RZ] += v * zv;
        }
    };
    // two elements per trip with all loads issued first (load latency)
    const long long G = (long long)gridDim.x * blockDim.x;
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    for (; i + G < n; i += 2 * G) {
        const long long j = i + G;
        const double s1i = s1v[i], s1j = s1v[j], s2i = s2v[i], s2j = s2v[j];
        const double ai = z1[i], aj = z1[j], di = z2[i], dj = z2[j];
        const double xai = step ? (double)dba[i] : 0.0, xaj = step ? (double)dba[j] : 0.0;
        const double xi = step ? (double)db[i] : 0.0, xj = step ? (double)db[j] : 0.0;
        const double bei = beta[i], bej = beta[j], qi = Qb[i], qj = Qb[j], bbi = b[i], bbj = b[j];
        elem(i, s1i, s2i, ai, di, xai, xi, bei, qi, bbi);
        elem(j, s1j, s2j, aj, dj, xaj, xj, bej, qj, bbj);
    }
    if (i < n)
        elem(i, s1v[i], s2v[i], z1[i], z2[i], step ? (double)dba[i] : 0.0, step ? (double)db[i] : 0.0, beta[i], Qb[i],
             b[i]);
    if (grid_reduce<RR_N>(acc, ws, RR_MAXMASK, 0u) && csc && threadIdx.x == 0) cg_start(csc, ws.out[RR_RZ], 0.0, crtol);
}
template <typename TV, typename TD>
static __global__ void __launch_bounds__(EW_THREADS, 3)
ipm_resdiag_kernel(long long n, const double* __restrict__ b, const double* __restrict__ Qb, double lam,
                   const double* __restrict__ beta, double* __restrict__ s1v, double* __restrict__ s2v,
                   double* __restrict__ z1, double* __restrict__ z2, const TD* __restrict__ dba,
                   const TD* __restrict__ db, const double* __restrict__ sigmu_p,
                   const double* __restrict__ alpha_p, double* __restrict__ rd, double* __restrict__ Db,
                   double* __restrict__ Minv, TV* __restrict__ Db_lo, TV* __restrict__ Minv_lo, int precond,
                   double* __restrict__ rhs, RedWorkspace ws, TV* __restrict__ cr, TV* __restrict__ cp,
                   CgScalars* csc, DevScalar crtol) {
    ipm_resdiag_kernel_body<TV, TD>(n, b, Qb, lam, beta, s1v, s2v, z1, z2, dba, db, sigmu_p, alpha_p, rd, Db, Minv, Db_lo, Minv_lo, precond, rhs, ws, cr, cp, csc, crtol);
}

// FP64 barrier diagonals alone (mixed precision at loose Newton tolerances
// skips them in the residual pass; the first FP64 product or FP64 fallback
// of the iteration computes them here)
static __global__ void ipm_diag64_kernel(long long n, const double* __restrict__ s1, const double* __restrict__ s2,
                                         const double* __restrict__ z1, const double* __restrict__ z2,
                                         double* __restrict__ Db, double* __restrict__ Minv, int precond) {
    CSIPM_GRID_LOOP(i, n) {
        const ElemDiag g = elem_diag(s1[i], s2[i], z1[i], z2[i], precond);   // as in ipm_resdiag_kernel
        Db[i] = g.db;
        Minv[i] = g.mi;
    }
}

// beta += alpha db (the slacks and multipliers take their step in the next
// residual pass)
template <typename TD>
__device__ __forceinline__ void ipm_beta_step_kernel_body(long long n, double* __restrict__ beta, const TD* __restrict__ db,
                                            const double* __restrict__ alpha_p) {
    const double alpha = *alpha_p;
    CSIPM_GRID_LOOP(i, n) beta[i] += alpha * (double)db[i];
}
template <typename TD>
static __global__ void ipm_beta_step_kernel(long long n, double* __restrict__ beta, const TD* __restrict__ db,
                                            const double* __restrict__ alpha_p) {
    ipm_beta_step_kernel_body<TD>(n, beta, db, alpha_p);
}

// c = (s1 + s2)/2
__device__ __forceinline__ void half_sum_kernel_body(long long n, const double* __restrict__ s1, const double* __restrict__ s2,
                                       double* __restrict__ c) {
    CSIPM_GRID_LOOP(i, n) c[i] = 0.5 * (s1[i] + s2[i]);
}
static __global__ void half_sum_kernel(long long n, const double* __restrict__ s1, const double* __restrict__ s2,
                                       double* __restrict__ c) {
    half_sum_kernel_body(n, s1, s2, c);
}

// ------------------------------------------------------------------ utilities
template <typename TA, typename TB>
static __global__ void convert_kernel(long long n, const TA* __restrict__ a, TB* __restrict__ b) {
    CSIPM_GRID_LOOP(i, n) b[i] = (TB)a[i];
}

static __global__ void axpy_kernel(long long n, double alpha, const double* __restrict__ x, double* __restrict__ y) {
    CSIPM_GRID_LOOP(i, n) y[i] += alpha * x[i];
}

// y = x - y  (residual r = rhs - Kx in place on y)
static __global__ void sub_from_kernel(long long n, const double* __restrict__ x, double* __restrict__ y) {
    CSIPM_GRID_LOOP(i, n) y[i] = x[i] - y[i];
}

// dot products on the device
static __global__ void dot2_kernel(long long n, const double* __restrict__ a, const double* __restrict__ b,
                            const double* __restrict__ c2, const double* __restrict__ d2, RedWorkspace ws) {
    double acc[2] = {0.0, 0.0};
    CSIPM_GRID_LOOP(i, n) {
        acc[0] += a[i] * b[i];
        if (c2) acc[1] += c2[i] * d2[i];
    }
    grid_reduce<2>(acc, ws, 0u, 0u);
}

// ------------------------------------------------------------------ NLPModels / KKT plugin
// g = [AtA beta - Atz0 ; lambda] (beta part fused in the operator epilogue)
struct EpiGrad {
    const double* b;
    double* g;
    using Pre = NoPre;
    __device__ __forceinline__ NoPre pre(int) const { return {}; }
    __device__ __forceinline__ void put(int l, double v, const NoPre&) { g[l] = v - b[l]; }
    __device__ __forceinline__ void finish() {}
};

static __global__ void fill_kernel(long long n, double v, double* __restrict__ y) {
    CSIPM_GRID_LOOP(i, n) y[i] = v;
}

static __global__ void fill_f32_kernel(long long n, float v, float* __restrict__ y) {
    CSIPM_GRID_LOOP(i, n) y[i] = v;
}

// cons!: c = [-beta - c ; beta - c]   (src/fft_model.jl:91-101)
static __global__ void cons_kernel(long long n, const double* __restrict__ x, double* __restrict__ out) {
    CSIPM_GRID_LOOP(i, n) {
        const double be = x[i], ce = x[n + i];
        out[i] = -be - ce;
        out[n + i] = be - ce;
    }
}

// hprod: hv = w [AtA v_b ; 0]
struct EpiScale {
    double w;
    double* out;
    using Pre = NoPre;
    __device__ __forceinline__ NoPre pre(int) const { return {}; }
    __device__ __forceinline__ void put(int l, double v, const NoPre&) { out[l] = w * v; }
    __device__ __forceinline__ void finish() {}
};

// build_kkt!  (src/fft_kkt.jl:285-307)
static __global__ void kkt_build_kernel(long long n, const double* __restrict__ pr_diag, double* __restrict__ L1,
                                 double* __restrict__ L2, double* __restrict__ P11, double* __restrict__ P12,
                                 double* __restrict__ P22) {
    CSIPM_GRID_LOOP(i, n) {
        const double S1 = pr_diag[2 * n + i], S2 = pr_diag[3 * n + i];
        const double l1 = S1 + S2, l2 = S1 - S2;
        const double Minv = 1.0 / (1.0 + l1);
        const double S = 1.0 / (l1 - l2 * l2 * Minv);
        L1[i] = l1;
        L2[i] = l2;
        P22[i] = S;
        P12[i] = -l2 * S * Minv;
        P11[i] = Minv + Minv * l2 * S * l2 * Minv;
    }
}

// condensed mul!  yb = beta*yb + alpha*(AtA xb + L1 xb + L2 xz), yz = beta*yz + alpha*(L2 xb + L1 xz)
// (src/fft_kkt.jl:27-44); the AtA part arrives through the operator epilogue.
struct EpiCondensed {
    const double* x;    // 2N
    double* y;          // 2N
    const double* L1;
    const double* L2;
    long long n;
    double alpha, beta;
    using Pre = NoPre;
    __device__ __forceinline__ NoPre pre(int) const { return {}; }
    __device__ __forceinline__ void put(int l, double v, const NoPre&) {
        const double xb = x[l], xz = x[n + l];
        const double l1 = L1[l], l2 = L2[l];
        y[l] = beta * y[l] + alpha * (v + l1 * xb + l2 * xz);
        y[n + l] = beta * y[n + l] + alpha * (l2 * xb + l1 * xz);
    }
    __device__ __forceinline__ void finish() {}
};

// preconditioner mul!  (src/fft_kkt.jl:73-85)
static __global__ void precond_mul_kernel(long long n, double* __restrict__ y, const double* __restrict__ x,
                                   const double* __restrict__ P11, const double* __restrict__ P12,
                                   const double* __restrict__ P22, double alpha, double beta) {
    CSIPM_GRID_LOOP(i, n) {
        const double xb = x[i], xz = x[n + i];
        y[i] = beta * y[i] + alpha * (P11[i] * xb + P12[i] * xz);
        y[n + i] = beta * y[n + i] + alpha * (P12[i] * xb + P22[i] * xz);
    }
}

// full KKT mul! body (src/fft_kkt.jl:223-246) fused into the operator epilogue
struct EpiKKT {
    const double* x;    // 6N
    double* y;          // 6N
    long long n;
    double alpha, beta;
    using Pre = NoPre;
    __device__ __forceinline__ NoPre pre(int) const { return {}; }
    __device__ __forceinline__ void put(int l, double v, const NoPre&) {
        const long long N = n;
        const double xb = x[l], xz = x[N + l], xs1 = x[2 * N + l], xs2 = x[3 * N + l];
        const double xy1 = x[4 * N + l], xy2 = x[5 * N + l];
        y[l] = beta * y[l] + alpha * (v - xy1 + xy2);
        y[N + l] = beta * y[N + l] - alpha * (xy1 + xy2);
        y[2 * N + l] = beta * y[2 * N + l] - alpha * xy1;
        y[3 * N + l] = beta * y[3 * N + l] - alpha * xy2;
        y[4 * N + l] = beta * y[4 * N + l] + alpha * (-xb - xz - xs1);
        y[5 * N + l] = beta * y[5 * N + l] + alpha * (xb - xz - xs2);
    }
    __device__ __forceinline__ void finish() {}
};

// jtprod!  (src/fft_kkt.jl:253-275)
static __global__ void jtprod_kernel(long long n, double* __restrict__ y, const double* __restrict__ x) {
    CSIPM_GRID_LOOP(i, n) {
        const double y1 = x[i], y2 = x[n + i];
        y[i] = -y1 + y2;
        y[n + i] = -y1 - y2;
        y[2 * n + i] = -y1;
        y[3 * n + i] = -y2;
    }
}

// solve_kkt! right-hand side (src/fft_kkt.jl:334-335): b = [w1 - w3 + w4 - S1 w5 + S2 w6 ; w2 - w3 - w4 - S1 w5 - S2 w6]
static __global__ void kkt_rhs_kernel(long long n, const double* __restrict__ w, const double* __restrict__ pr_diag,
                               double* __restrict__ b) {
    CSIPM_GRID_LOOP(i, n) {
        const double S1 = pr_diag[2 * n + i], S2 = pr_diag[3 * n + i];
        const double w1 = w[i], w2 = w[n + i], w3 = w[2 * n + i], w4 = w[3 * n + i], w5 = w[4 * n + i], w6 = w[5 * n + i];
        b[i] = w1 - w3 + w4 - S1 * w5 + S2 * w6;
        b[n + i] = w2 - w3 - w4 - S1 * w5 - S2 * w6;
    }
}

// solve_kkt! back-substitution (src/fft_kkt.jl:345-350)
static __global__ void kkt_back_kernel(long long n, double* __restrict__ w, const double* __restrict__ x,
                                const double* __restrict__ pr_diag) {
    CSIPM_GRID_LOOP(i, n) {
        const double S1 = pr_diag[2 * n + i], S2 = pr_diag[3 * n + i];
        const double w1 = x[i], w2 = x[n + i];
        double w3 = w[2 * n + i], w4 = w[3 * n + i], w5 = w[4 * n + i], w6 = w[5 * n + i];
        w5 = -(w3 + S1 * (w1 + w2 + w5));
        w6 = -(w4 + S2 * (-w1 + w2 + w6));
        w3 = (w3 + w5) / S1;
        w4 = (w4 + w6) / S2;
        w[i] = w1; w[n + i] = w2; w[2 * n + i] = w3; w[3 * n + i] = w4; w[4 * n + i] = w5; w[5 * n + i] = w6;
    }
}

// ---- 2N PCG of the KKT plugin (Krylov.jl cg semantics, M = block preconditioner)
// z = P r (2x2 blocks), written into z; returns r.z
__device__ __forceinline__ void pblock(const double* P11, const double* P12, const double* P22, long long i,
                                       double rb, double rz, double& zb, double& zz) {
    if (P11) {
        zb = P11[i] * rb + P12[i] * rz;
        zz = P12[i] * rb + P22[i] * rz;
    } else {
        zb = rb;
        zz = rz;
    }
}

// x = 0, r = b, p = z = P r, rz = r.z
static __global__ void kcg_init_kernel(long long n, const double* __restrict__ b, double* __restrict__ x, double* __restrict__ r,
                                double* __restrict__ p, const double* __restrict__ P11, const double* __restrict__ P12,
                                const double* __restrict__ P22, RedWorkspace ws, CgScalars* sc, double atol, double rtol) {
    double acc[1] = {0.0};
    CSIPM_GRID_LOOP(i, n) {
        const double rb = b[i], rzv = b[n + i];
        double zb, zz;
        pblock(P11, P12, P22, i, rb, rzv, zb, zz);
        x[i] = 0.0; x[n + i] = 0.0;
        r[i] = rb; r[n + i] = rzv;
        p[i] = zb; p[n + i] = zz;
        acc[0] += rb * zb + rzv * zz;
    }
    if (grid_reduce<1>(acc, ws, 0u, 0u) && threadIdx.x == 0) {
        const double rz = ws.out[0];
        sc->rz[0] = rz;
        sc->rz0 = rz;
        sc->thresh = atol + rtol * sqrt(rz);
        sc->iters = 0;
        sc->breakdown = 0;
        sc->done = (sqrt(rz) <= sc->thresh) ? 1 : 0;
    }
}

// q = K p fused: qb = AtA pb + L1 pb + L2 pz ; qz = L2 pb + L1 pz ; acc p.q
struct EpiKcg {
    const double* p;
    double* q;
    const double* L1;
    const double* L2;
    long long n;
    RedWorkspace ws;
    double acc;
    struct Pre { double pb, pz, l1, l2; };
    __device__ __forceinline__ Pre pre(int l) const { return Pre{p[l], p[n + l], L1[l], L2[l]}; }
    __device__ __forceinline__ void put(int l, double v, const Pre& r) {
        const double pb = r.pb, pz = r.pz;
        const double l1 = r.l1, l2 = r.l2;
        const double qb = v + l1 * pb + l2 * pz;
        const double qz = l2 * pb + l1 * pz;
        q[l] = qb;
        q[n + l] = qz;
        acc += pb * qb + pz * qz;
    }
    __device__ __forceinline__ void finish() {
        double a[1] = {acc};
        grid_reduce<1>(a, ws, 0u, 0u);
    }
};

static __global__ void kcg_update_kernel(long long n, int it, double* __restrict__ x, double* __restrict__ r,
                                  const double* __restrict__ p, const double* __restrict__ q,
                                  const double* __restrict__ P11, const double* __restrict__ P12,
                                  const double* __restrict__ P22, RedWorkspace ws, CgScalars* sc) {
    if (sc->done) return;
    const double pq = sc->pq;
    const double alpha = sc->rz[it & 1] / pq;
    double acc[1] = {0.0};
    CSIPM_GRID_LOOP(i, n) {
        x[i] += alpha * p[i];
        x[n + i] += alpha * p[n + i];
        const double rb = r[i] - alpha * q[i];
        const double rzv = r[n + i] - alpha * q[n + i];
        r[i] = rb;
        r[n + i] = rzv;
        double zb, zz;
        pblock(P11, P12, P22, i, rb, rzv, zb, zz);
        acc[0] += rb * zb + rzv * zz;
    }
    if (grid_reduce<1>(acc, ws, 0u, 0u) && threadIdx.x == 0) {
        const double rzn = ws.out[0];
        sc->rz[(it + 1) & 1] = rzn;
        sc->iters += 1;     // counted on the device: graph replays reuse the same `it` values
        if (!isfinite(rzn)) { sc->breakdown = 1; sc->done = 1; }
        else if (sqrt(rzn) <= sc->thresh) sc->done = 1;
    }
}

static __global__ void kcg_pupdate_kernel(long long n, int it, const double* __restrict__ r, double* __restrict__ p,
                                   const double* __restrict__ P11, const double* __restrict__ P12,
                                   const double* __restrict__ P22, const CgScalars* sc) {
    if (sc->done) return;
    const double b = sc->rz[(it + 1) & 1] / sc->rz[it & 1];
    CSIPM_GRID_LOOP(i, n) {
        double zb, zz;
        pblock(P11, P12, P22, i, r[i], r[n + i], zb, zz);
        p[i] = zb + b * p[i];
        p[n + i] = zz + b * p[n + i];
    }
}

}  // namespace csipm
