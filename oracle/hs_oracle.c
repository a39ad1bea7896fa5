/*
 * CPU oracle for the HybridSmoothers.jl preconditioner-apply path — TEST
 * INFRASTRUCTURE ONLY (see hs_oracle_tmpl.h for the contract).  Built into
 * oracle/libhsoracle.so by oracle/Makefile with -ffp-contract=off; loaded by
 * oracle/hs_oracle.py for tests, smoke() and the CPU-baseline arm of bench.py.
 * The product library (libhsb200.so) never links or calls it.
 *
 * Parity status: pinned.  The L1GS and Chebyshev restatements reproduce every
 * known-answer vector in the reference's test suite
 * (test/test_preconditioners.jl, test/test_chebyshev.jl, test/gpu/gpu.jl) and
 * the a* table of src/chebyshev.jl:208-210; tests/test_oracle_kat.py checks
 * them.  The Krylov drivers (PCG, restarted GMRES) stand in for Krylov.jl,
 * which the reference reaches through LinearSolve.jl and does not vendor:
 * their iteration counts are this oracle's own and are not pinned to Krylov.jl.
 * Their dot products are compensated (Dot2) and every update separately
 * rounded, the arithmetic the device drivers use.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define REAL double
#define SFX _f64
#define ABS(x) fabs(x)
#define SQRT(x) sqrt(x)
#include "hs_oracle_tmpl.h"
#undef REAL
#undef SFX
#undef ABS
#undef SQRT

#define REAL float
#define SFX _f32
#define ABS(x) fabsf(x)
#define SQRT(x) sqrtf(x)
#include "hs_oracle_tmpl.h"
#undef REAL
#undef SFX
#undef ABS
#undef SQRT

/* ------------------------------------------------------------------------ */
/* Krylov drivers (FP64 outer loop) with an L1GS or Chebyshev preconditioner */
/* whose arithmetic is FP64 or FP32 ("mixed": the smoother works on FP32     */
/* copies; the residual is rounded to FP32 on the way in and the correction  */
/* widened to FP64 on the way out).                                          */
/* ------------------------------------------------------------------------ */

typedef struct {
    int32_t type;   /* 0 none, 1 L1GS, 2 Chebyshev 4th kind, 3 Chebyshev 1st kind */
    int32_t fp32;   /* 1: smoother arithmetic in FP32 */
    /* L1GS */
    int32_t ps, sweep, kind;
    const void* SL;
    const void* SU;
    const void* D;
    const int32_t* rp;
    const int32_t* ci;
    const void* v;
    const int32_t* diag;
    /* Chebyshev (rp/ci/v above are the CSR matrix in the smoother precision) */
    const void* l1inv;
    double rho, astar;
    int32_t degree;
} hso_prec;

static void prec_apply(int32_t n, const hso_prec* P, const double* r, double* z)
{
    if (P == NULL || P->type == 0) {
        memcpy(z, r, sizeof(double) * (size_t)n);
        return;
    }
    if (!P->fp32) {
        if (P->type == 1) {
            hso_l1gs_apply_f64(n, P->ps, P->sweep, P->kind, (const double*)P->SL,
                               (const double*)P->SU, P->rp, P->ci, (const double*)P->v, P->diag,
                               (const double*)P->D, r, z, 1, 1);
        } else {
            double* w = (double*)malloc(sizeof(double) * (size_t)n * 3);
            for (int32_t i = 0; i < n; ++i) z[i] = 0.0;
            if (P->type == 2)
                hso_cheb4_smooth_f64(n, P->rp, P->ci, (const double*)P->v, (const double*)P->l1inv,
                                     P->rho, P->degree, z, r, w, w + n);
            else
                hso_cheb1_smooth_f64(n, P->rp, P->ci, (const double*)P->v, (const double*)P->l1inv,
                                     P->rho, P->astar, P->degree, z, r, w, w + n, w + 2 * (size_t)n);
            free(w);
        }
        return;
    }
    float* rf = (float*)malloc(sizeof(float) * (size_t)n * 5);
    float* zf = rf + n;
    for (int32_t i = 0; i < n; ++i) rf[i] = (float)r[i];
    if (P->type == 1) {
        hso_l1gs_apply_f32(n, P->ps, P->sweep, P->kind, (const float*)P->SL, (const float*)P->SU,
                           P->rp, P->ci, (const float*)P->v, P->diag, (const float*)P->D, rf, zf, 1, 1);
    } else {
        float* w = zf + n;
        for (int32_t i = 0; i < n; ++i) zf[i] = 0.0f;
        if (P->type == 2)
            hso_cheb4_smooth_f32(n, P->rp, P->ci, (const float*)P->v, (const float*)P->l1inv, P->rho,
                                 P->degree, zf, rf, w, w + n);
        else
            hso_cheb1_smooth_f32(n, P->rp, P->ci, (const float*)P->v, (const float*)P->l1inv, P->rho,
                                 P->astar, P->degree, zf, rf, w, w + n, w + 2 * (size_t)n);
    }
    for (int32_t i = 0; i < n; ++i) z[i] = (double)zf[i];
    free(rf);
}

/*
 * Compensated dot product (Ogita, Rump & Oishi 2005, "Dot2"): TwoProduct via
 * fma, TwoSum, errors accumulated separately.  As accurate as a dot in twice
 * the working precision, so its rounded value does not depend on the order in
 * which a parallel reduction meets the terms; the device drivers use the same
 * accumulation, which is what lets their iterates match these.
 */
static double dot(int32_t n, const double* a, const double* b)
{
    double s = 0.0, c = 0.0;
    for (int32_t i = 0; i < n; ++i) {
        const double p = a[i] * b[i];
        const double pe = fma(a[i], b[i], -p);
        const double t = s + p;
        const double bb = t - s;
        const double q = (s - (t - bb)) + (p - bb);
        s = t;
        c = c + (q + pe);
    }
    return s + c;
}

/*
 * Preconditioned CG (Hestenes-Stiefel), x0 = 0, stop when the recursive
 * residual satisfies sqrt(r.r) <= rtol*sqrt(b.b).  Every vector update is two
 * rounded operations (the file is built with -ffp-contract=off).  Returns the
 * iteration count (number of A*p products), or -1 if maxit was reached;
 * *relres receives the true relative residual ||b - A x||/||b|| of x.
 */
int32_t hso_pcg(int32_t n, const int32_t* rp, const int32_t* ci, const double* v, const double* b,
                double* x, const hso_prec* P, double rtol, int32_t maxit, double* relres)
{
    double* r = (double*)malloc(sizeof(double) * (size_t)n * 4);
    double* z = r + n;
    double* p = z + n;
    double* q = p + n;
    for (int32_t i = 0; i < n; ++i) { x[i] = 0.0; r[i] = b[i]; }
    const double bb = dot(n, b, b);
    const double bnorm = sqrt(bb);
    int32_t it = 0, conv = 0;
    if (bb == 0.0) { conv = 1; goto done; }
    prec_apply(n, P, r, z);
    memcpy(p, z, sizeof(double) * (size_t)n);
    double rz = dot(n, r, z);
    for (it = 1; it <= maxit; ++it) {
        hso_spmv_f64(n, rp, ci, v, p, q);
        const double alpha = rz / dot(n, p, q);
        for (int32_t i = 0; i < n; ++i) { x[i] = x[i] + alpha * p[i]; r[i] = r[i] - alpha * q[i]; }
        const double rr = dot(n, r, r);
        if (sqrt(rr) <= rtol * bnorm) { conv = 1; break; }
        prec_apply(n, P, r, z);
        const double rz_new = dot(n, r, z);
        const double beta = rz_new / rz;
        rz = rz_new;
        for (int32_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    }
done:
    hso_spmv_f64(n, rp, ci, v, x, q);
    {
        double ss = 0.0;
        for (int32_t i = 0; i < n; ++i) { double d = b[i] - q[i]; ss += d * d; }
        *relres = bnorm > 0 ? sqrt(ss) / bnorm : 0.0;
    }
    free(r);
    if (!conv) return -1;
    return it > maxit ? maxit : it;
}

/*
 * Restarted GMRES(m), right preconditioned (A M^-1 u = b, x = M^-1 u), x0 = 0,
 * classical Gram-Schmidt applied twice (CGS2: all projections of a pass from
 * the same w, then w -= sum_i h_i V_i in order i = 0..j), Givens rotations.
 * A cycle ends when |g_{j+1}| <= rtol*||b||; the restart residual is
 * r = b - A x (term by term, as five-argument mul!) and convergence is
 * ||r|| <= rtol*||b||.  Returns total inner iterations or -1.
 */
int32_t hso_gmres(int32_t n, const int32_t* rp, const int32_t* ci, const double* v, const double* b,
                  double* x, const hso_prec* P, int32_t m, double rtol, int32_t maxit,
                  double* relres)
{
    double* V = (double*)malloc(sizeof(double) * (size_t)n * (m + 1));
    double* w = (double*)malloc(sizeof(double) * (size_t)n * 3);
    double* u = w + n;
    double* r = u + n;
    double* H = (double*)calloc((size_t)(m + 1) * m, sizeof(double));
    double* cs = (double*)calloc((size_t)m, sizeof(double));
    double* sn = (double*)calloc((size_t)m, sizeof(double));
    double* g = (double*)calloc((size_t)m + 1, sizeof(double));
    double* yv = (double*)calloc((size_t)m, sizeof(double));
    double* hcol = (double*)calloc((size_t)m + 1, sizeof(double));
#define HH(i, j) H[(size_t)(i) * m + (j)]
    for (int32_t i = 0; i < n; ++i) { x[i] = 0.0; r[i] = b[i]; }
    const double bnorm = sqrt(dot(n, b, b));
    const double tol = rtol * bnorm;
    double beta = bnorm;
    int32_t total = 0, conv = 0;
    if (bnorm == 0.0) { conv = 1; goto out; }
    while (total < maxit) {
        for (int32_t i = 0; i < n; ++i) V[i] = r[i] / beta;
        memset(H, 0, sizeof(double) * (size_t)(m + 1) * m);
        for (int32_t i = 0; i <= m; ++i) g[i] = 0.0;
        g[0] = beta;
        int32_t jend = 0;
        for (int32_t j = 0; j < m; ++j) {
            prec_apply(n, P, V + (size_t)j * n, u);
            hso_spmv_f64(n, rp, ci, v, u, w);
            for (int32_t pass = 0; pass < 2; ++pass) {
                for (int32_t i = 0; i <= j; ++i) hcol[i] = dot(n, V + (size_t)i * n, w);
                for (int32_t t = 0; t < n; ++t) {
                    double s = w[t];
                    for (int32_t i = 0; i <= j; ++i) s = s - hcol[i] * V[(size_t)i * n + t];
                    w[t] = s;
                }
                for (int32_t i = 0; i <= j; ++i) HH(i, j) = HH(i, j) + hcol[i];
            }
            const double hn = sqrt(dot(n, w, w));
            HH(j + 1, j) = hn;
            if (hn != 0.0)
                for (int32_t t = 0; t < n; ++t) V[(size_t)(j + 1) * n + t] = w[t] / hn;
            for (int32_t i = 0; i < j; ++i) {
                const double a0 = HH(i, j), a1 = HH(i + 1, j);
                HH(i, j) = cs[i] * a0 + sn[i] * a1;
                HH(i + 1, j) = -sn[i] * a0 + cs[i] * a1;
            }
            const double a0 = HH(j, j), a1 = HH(j + 1, j);
            const double den = sqrt(a0 * a0 + a1 * a1);
            cs[j] = den == 0.0 ? 1.0 : a0 / den;
            sn[j] = den == 0.0 ? 0.0 : a1 / den;
            HH(j, j) = cs[j] * a0 + sn[j] * a1;
            HH(j + 1, j) = 0.0;
            g[j + 1] = -sn[j] * g[j];
            g[j] = cs[j] * g[j];
            ++total;
            jend = j + 1;
            if (fabs(g[j + 1]) <= tol || hn == 0.0 || total >= maxit) break;
        }
        for (int32_t i = jend - 1; i >= 0; --i) {
            double s = g[i];
            for (int32_t t = i + 1; t < jend; ++t) s = s - HH(i, t) * yv[t];
            yv[i] = s / HH(i, i);
        }
        for (int32_t t = 0; t < n; ++t) {
            double s = 0.0;
            for (int32_t i = 0; i < jend; ++i) s = s + yv[i] * V[(size_t)i * n + t];
            w[t] = s;
        }
        prec_apply(n, P, w, u);
        for (int32_t t = 0; t < n; ++t) x[t] = x[t] + u[t];
        for (int32_t t = 0; t < n; ++t) r[t] = b[t];
        hso_spmv_sub_f64(n, rp, ci, v, x, r);
        beta = sqrt(dot(n, r, r));
        if (beta <= tol) { conv = 1; break; }
    }
out:
    *relres = bnorm > 0 ? beta / bnorm : 0.0;
#undef HH
    free(V); free(w); free(H); free(cs); free(sn); free(g); free(yv); free(hcol);
    return conv ? total : -1;
}

int32_t hso_omp_max_threads(void)
{
#ifdef _OPENMP
    extern int omp_get_max_threads(void);
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void hso_omp_set_threads(int32_t t)
{
#ifdef _OPENMP
    extern void omp_set_num_threads(int);
    omp_set_num_threads(t);
#else
    (void)t;
#endif
}
