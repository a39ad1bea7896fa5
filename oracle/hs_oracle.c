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
 * them.  Two pairs of Krylov drivers: hso_cg_kjl / hso_gmres_kjl restate
 * Krylov.jl's cg and gmres as the reference calls them through LinearSolve.jl
 * (Krylov.jl is not vendored: restated from its published algorithms, the
 * reference's call sites test/test_preconditioners.jl:65,93 and README.md:29);
 * hso_pcg / hso_gmres are this project's own drivers (true-residual stopping,
 * CGS2).  Dot products are compensated (Dot2) and every update separately
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

/* ------------------------------------------------------------------------ */
/* Krylov.jl's CG and GMRES as LinearSolve.jl's KrylovJL_CG / KrylovJL_GMRES */
/* call them with Pl = P (test/test_preconditioners.jl:65,93): M = P applied */
/* with ldiv! (z = P \ r), x0 = 0, stopping at rNorm <= atol + rtol*rNorm0.  */
/* Restated from the published algorithms of Krylov.jl (0.9/0.10, src/cg.jl  */
/* and src/gmres.jl; not vendored in the reference).  Dot products and norms */
/* are the compensated sums above (Krylov.jl calls BLAS, whose summation     */
/* order is the library's own); updates are separately rounded.              */
/* ------------------------------------------------------------------------ */

/*
 * cg!: r = b, z = M \ r, p = z, gamma = r.z, rNorm = sqrt(gamma),
 * eps = atol + rtol*rNorm; each iteration q = A p, alpha = gamma / p.q,
 * x += alpha p, r -= alpha q, z = M \ r, gamma' = r.z, rNorm = sqrt(gamma');
 * stop when rNorm <= eps (or rNorm + 1 <= 1), else p = z + (gamma'/gamma) p.
 * A non-positive p.q (zero or negative curvature) stops without convergence.
 * itmax 0 means 2n.  Returns the iteration count (Krylov.jl's niter), or -1
 * when not solved; *relres = ||b - A x|| / ||b||, *rnorm = the final rNorm.
 */
int32_t hso_cg_kjl(int32_t n, const int32_t* rp, const int32_t* ci, const double* v, const double* b, double* x,
                   const hso_prec* P, double atol, double rtol, int32_t itmax, double* relres, double* rnorm)
{
    double* r = (double*)malloc(sizeof(double) * (size_t)n * 4);
    double* z = r + n;
    double* p = z + n;
    double* q = p + n;
    if (itmax <= 0) itmax = 2 * n;
    for (int32_t i = 0; i < n; ++i) { x[i] = 0.0; r[i] = b[i]; }
    prec_apply(n, P, r, z);
    memcpy(p, z, sizeof(double) * (size_t)n);
    double gamma = dot(n, r, z);
    double rn = sqrt(gamma);
    const double eps = atol + rtol * rn;
    int32_t iter = 0, solved = (gamma == 0.0) || (rn <= eps), failed = 0;
    while (!solved && iter < itmax) {
        hso_spmv_f64(n, rp, ci, v, p, q);
        const double pq = dot(n, p, q);
        if (!(pq > 0.0)) { failed = 1; break; }
        const double alpha = gamma / pq;
        for (int32_t i = 0; i < n; ++i) { x[i] = x[i] + alpha * p[i]; r[i] = r[i] - alpha * q[i]; }
        prec_apply(n, P, r, z);
        const double gnew = dot(n, r, z);
        rn = sqrt(gnew);
        ++iter;
        solved = (rn <= eps) || (rn + 1.0 <= 1.0);
        if (!solved) {
            const double beta = gnew / gamma;
            gamma = gnew;
            for (int32_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
        }
    }
    const double bnorm = sqrt(dot(n, b, b));
    hso_spmv_f64(n, rp, ci, v, x, q);
    for (int32_t i = 0; i < n; ++i) q[i] = b[i] - q[i];
    *relres = bnorm > 0 ? sqrt(dot(n, q, q)) / bnorm : 0.0;
    *rnorm = rn;
    free(r);
    return (solved && !failed) ? iter : -1;
}

/*
 * Symmetric Givens reflection [c s; s -c] [a; b] = [rho; 0] (the stable
 * form of Golub & Van Loan / Bindel, Demmel & Kahan that Krylov.jl's
 * sym_givens computes).
 */
static void sym_givens(double a, double b, double* c, double* s, double* rho)
{
    if (b == 0.0) {
        *c = (a == 0.0) ? 1.0 : copysign(1.0, a);
        *s = 0.0;
        *rho = fabs(a);
    } else if (a == 0.0) {
        *c = 0.0;
        *s = copysign(1.0, b);
        *rho = fabs(b);
    } else if (fabs(b) > fabs(a)) {
        const double t = a / b;
        *s = copysign(1.0, b) / sqrt(1.0 + t * t);
        *c = *s * t;
        *rho = b / *s;
    } else {
        const double t = b / a;
        *c = copysign(1.0, a) / sqrt(1.0 + t * t);
        *s = *c * t;
        *rho = a / *c;
    }
}

/*
 * gmres! with restart = true and memory m, left preconditioner M:
 * r0 = M \ (b - A x) (x = 0 first), beta = ||r0||, eps = atol + rtol*beta0.
 * A cycle sets z_1 = beta, V_1 = r0 / beta; inner iteration k: q = M \ (A V_k),
 * modified Gram-Schmidt R_ik = V_i.q, q -= R_ik V_i (i = 1..k, in order),
 * Hbis = ||q||, the previous reflections applied to column k of R, a new one
 * from sym_givens(R_kk, Hbis), zeta_{k+1} = s_k z_k, z_k = c_k z_k,
 * rNorm = |zeta_{k+1}|; the cycle ends when rNorm <= eps (or rNorm + 1 <= 1),
 * k = m, the iteration cap, or breakdown (Hbis <= btol = eps(double)^(3/4));
 * otherwise V_{k+1} = q / Hbis, z_{k+1} = zeta_{k+1}.  Then y = R \ z by back
 * substitution (columns from the last; y_i = 0 where |R_ii| <= btol) and
 * x += sum_i y_i V_i.  Returns niter (total inner iterations) or -1.
 */
int32_t hso_gmres_kjl(int32_t n, const int32_t* rp, const int32_t* ci, const double* v, const double* b, double* x,
                      const hso_prec* P, int32_t m, double atol, double rtol, int32_t itmax, double* relres,
                      double* rnorm)
{
    const double btol = pow(2.220446049250313e-16, 0.75);
    double* V = (double*)malloc(sizeof(double) * (size_t)n * (m + 1));
    double* w = (double*)malloc(sizeof(double) * (size_t)n * 3);
    double* q = w + n;
    double* xr = q + n;
    double* R = (double*)calloc((size_t)(m + 1) * m, sizeof(double));
    double* c = (double*)calloc((size_t)m, sizeof(double));
    double* s = (double*)calloc((size_t)m, sizeof(double));
    double* z = (double*)calloc((size_t)m + 1, sizeof(double));
    double* yv = (double*)calloc((size_t)m, sizeof(double));
#define RR(i, j) R[(size_t)(i) * m + (j)]
    if (itmax <= 0) itmax = 2 * n;
    for (int32_t i = 0; i < n; ++i) x[i] = 0.0;
    prec_apply(n, P, b, V);   /* r0 = M \ b, in V_1's storage */
    double beta = sqrt(dot(n, V, V));
    double rn = beta;
    const double eps = atol + rtol * rn;
    int32_t iter = 0, npass = 0, solved = rn <= eps, breakdown = 0;
    while (!(solved || iter >= itmax || breakdown)) {
        memset(R, 0, sizeof(double) * (size_t)(m + 1) * m);
        memset(z, 0, sizeof(double) * (size_t)(m + 1));
        if (npass >= 1) {
            hso_spmv_f64(n, rp, ci, v, x, w);
            for (int32_t i = 0; i < n; ++i) w[i] = b[i] - w[i];
            prec_apply(n, P, w, V);
            beta = sqrt(dot(n, V, V));
        }
        z[0] = beta;
        for (int32_t i = 0; i < n; ++i) V[i] = V[i] / beta;
        ++npass;
        int32_t k = 0;
        int32_t inner_done = 0;
        while (!inner_done) {
            const double* Vk = V + (size_t)k * n;
            hso_spmv_f64(n, rp, ci, v, Vk, w);
            prec_apply(n, P, w, q);
            for (int32_t i = 0; i <= k; ++i) {
                const double* Vi = V + (size_t)i * n;
                const double h = dot(n, Vi, q);
                RR(i, k) = h;
                for (int32_t t = 0; t < n; ++t) q[t] = q[t] - h * Vi[t];
            }
            const double hbis = sqrt(dot(n, q, q));
            for (int32_t i = 0; i < k; ++i) {
                const double tmp = c[i] * RR(i, k) + s[i] * RR(i + 1, k);
                RR(i + 1, k) = s[i] * RR(i, k) - c[i] * RR(i + 1, k);
                RR(i, k) = tmp;
            }
            sym_givens(RR(k, k), hbis, &c[k], &s[k], &RR(k, k));
            const double zeta = s[k] * z[k];
            z[k] = c[k] * z[k];
            rn = fabs(zeta);
            ++iter;
            ++k;
            solved = (rn <= eps) || (rn + 1.0 <= 1.0);
            breakdown = hbis <= btol;
            inner_done = solved || breakdown || k >= m || iter >= itmax;
            if (!inner_done) {
                double* Vn = V + (size_t)k * n;
                for (int32_t t = 0; t < n; ++t) Vn[t] = q[t] / hbis;
                z[k] = zeta;
            }
        }
        for (int32_t i = k - 1; i >= 0; --i) {
            double yi = z[i];
            for (int32_t j = k - 1; j > i; --j) yi = yi - RR(i, j) * yv[j];
            yv[i] = fabs(RR(i, i)) <= btol ? 0.0 : yi / RR(i, i);
        }
        for (int32_t t = 0; t < n; ++t) xr[t] = 0.0;
        for (int32_t i = 0; i < k; ++i) {
            const double* Vi = V + (size_t)i * n;
            for (int32_t t = 0; t < n; ++t) xr[t] = xr[t] + yv[i] * Vi[t];
        }
        for (int32_t t = 0; t < n; ++t) x[t] = x[t] + xr[t];
    }
    const double bnorm = sqrt(dot(n, b, b));
    hso_spmv_f64(n, rp, ci, v, x, w);
    for (int32_t i = 0; i < n; ++i) w[i] = b[i] - w[i];
    *relres = bnorm > 0 ? sqrt(dot(n, w, w)) / bnorm : 0.0;
    *rnorm = rn;
#undef RR
    free(V); free(w); free(R); free(c); free(s); free(z); free(yv);
    return solved ? iter : -1;
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
