/*
 * foam_cpu.c -- the CPU path the reference plugin mirrors (test oracle and
 * the bench's CPU baseline): OpenFOAM v2506's FP64 PCG and PBiCGStab loops
 * with diagonal / DIC preconditioning, restated from their published
 * algorithm (OpenFOAM is a third-party dependency, not vendored with the
 * reference; the reference states that its driver "exactly mirrors the
 * built-in PCG/PBiCGStab", metalFoamSolver.H:15-21, and reuses their
 * normFactor / gSumMag / checkConvergence, metalFoamSolver.C:119-135).
 * Also: an FP64 Krylov solve to a tight L2 tolerance (the accuracy oracle)
 * and a row-parallel Amul.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define VSMALL 1.0e-300

void orc_amul_rows(int32_t n, const int32_t* low, const int32_t* upp,
                   const int32_t* ownStart, const int32_t* losort,
                   const int32_t* losortStart, const double* diag,
                   const double* upper, const double* lower, const double* x,
                   double* y, int32_t transpose, int32_t nthreads)
{
    if (!lower) lower = upper;
    const double* up = transpose ? lower : upper;
    const double* lo = transpose ? upper : lower;
    (void)nthreads;
#pragma omp parallel for schedule(static) num_threads(nthreads > 0 ? nthreads : 1) if (nthreads > 1)
    for (int32_t i = 0; i < n; ++i)
    {
        /* per-row order of lduMatrix::Amul's face loop: losort side first */
        double s = diag[i] * x[i];
        for (int32_t k = losortStart[i]; k < losortStart[i + 1]; ++k)
        {
            const int32_t f = losort[k];
            s += lo[f] * x[low[f]];
        }
        for (int32_t f = ownStart[i]; f < ownStart[i + 1]; ++f)
            s += up[f] * x[upp[f]];
        y[i] = s;
    }
}

static double sum_prod(int32_t n, const double* a, const double* b, int nt)
{
    double s = 0.0;
    if (nt > 1)
    {
#pragma omp parallel for reduction(+ : s) schedule(static) num_threads(nt)
        for (int32_t i = 0; i < n; ++i) s += a[i] * b[i];
    }
    else
    {
        for (int32_t i = 0; i < n; ++i) s += a[i] * b[i];
    }
    return s;
}

static double sum_mag(int32_t n, const double* a, int nt)
{
    double s = 0.0;
    if (nt > 1)
    {
#pragma omp parallel for reduction(+ : s) schedule(static) num_threads(nt)
        for (int32_t i = 0; i < n; ++i) s += fabs(a[i]);
    }
    else
    {
        for (int32_t i = 0; i < n; ++i) s += fabs(a[i]);
    }
    return s;
}

typedef struct
{
    int kind;
    int32_t n, nf;
    const int32_t *low, *upp;
    const double* upper;
    double* rD;
} precond_t;

static void precond_setup(precond_t* P, int kind, int32_t n, int32_t nf,
                          const int32_t* low, const int32_t* upp,
                          const double* diag, const double* upper)
{
    P->kind = kind;
    P->n = n;
    P->nf = nf;
    P->low = low;
    P->upp = upp;
    P->upper = upper;
    P->rD = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    for (int32_t i = 0; i < n; ++i) P->rD[i] = diag[i];
    if (kind == ORC_PRECOND_DIC)
    {
        /* DIC reciprocal diagonal: rD[u] -= upper^2 / rD[l] in face order */
        for (int32_t f = 0; f < nf; ++f)
            P->rD[upp[f]] -= upper[f] * upper[f] / P->rD[low[f]];
    }
    for (int32_t i = 0; i < n; ++i) P->rD[i] = 1.0 / P->rD[i];
}

static void precond_apply(const precond_t* P, double* wA, const double* rA,
                          int nt)
{
    const int32_t n = P->n;
    if (P->kind == ORC_PRECOND_NONE)
    {
        memcpy(wA, rA, sizeof(double) * (size_t)n);
        return;
    }
    if (nt > 1)
    {
#pragma omp parallel for schedule(static) num_threads(nt)
        for (int32_t i = 0; i < n; ++i) wA[i] = P->rD[i] * rA[i];
    }
    else
    {
        for (int32_t i = 0; i < n; ++i) wA[i] = P->rD[i] * rA[i];
    }
    if (P->kind == ORC_PRECOND_DIC)
    {
        const int32_t* l = P->low;
        const int32_t* u = P->upp;
        const double* up = P->upper;
        const double* rD = P->rD;
        for (int32_t f = 0; f < P->nf; ++f)
            wA[u[f]] -= rD[u[f]] * up[f] * wA[l[f]];
        for (int32_t f = P->nf - 1; f >= 0; --f)
            wA[l[f]] -= rD[l[f]] * up[f] * wA[u[f]];
    }
}

int orc_foam_pcg(int32_t n, int32_t nf, const int32_t* low,
                 const int32_t* upp, const int32_t* ownStart,
                 const int32_t* losort, const int32_t* losortStart,
                 const double* diag, const double* upper, double* psi,
                 const double* source, int32_t precond, double tolerance,
                 double relTol, int32_t maxIter, int32_t minIter,
                 int32_t nthreads, orc_foam_perf* perf)
{
    const int nt = nthreads > 1 ? nthreads : 1;
    memset(perf, 0, sizeof(*perf));
    const size_t nb = sizeof(double) * (size_t)(n > 0 ? n : 1);
    double* pA = (double*)malloc(nb);
    double* wA = (double*)malloc(nb);
    double* rA = (double*)malloc(nb);

    orc_amul_rows(n, low, upp, ownStart, losort, losortStart, diag, upper,
                  NULL, psi, wA, 0, nt);
    for (int32_t i = 0; i < n; ++i) rA[i] = source[i] - wA[i];
    orc_sumA(n, nf, low, upp, diag, upper, NULL, pA);
    const double normFactor = orc_normfactor(n, psi, source, wA, pA);
    perf->initialResidual = sum_mag(n, rA, nt) / normFactor;
    perf->finalResidual = perf->initialResidual;

    if (minIter > 0
        || !orc_check_convergence(tolerance, relTol, perf->initialResidual,
                                  perf->finalResidual))
    {
        precond_t P;
        precond_setup(&P, precond, n, nf, low, upp, diag, upper);
        double wArA = 1e20, wArAold;
        do
        {
            wArAold = wArA;
            precond_apply(&P, wA, rA, nt);
            wArA = sum_prod(n, wA, rA, nt);
            if (perf->nIterations == 0)
            {
                memcpy(pA, wA, nb);
            }
            else
            {
                const double beta = wArA / wArAold;
#pragma omp parallel for schedule(static) num_threads(nt) if (nt > 1)
                for (int32_t i = 0; i < n; ++i) pA[i] = wA[i] + beta * pA[i];
            }
            orc_amul_rows(n, low, upp, ownStart, losort, losortStart, diag,
                          upper, NULL, pA, wA, 0, nt);
            const double wApA = sum_prod(n, wA, pA, nt);
            if (fabs(wApA) / normFactor < VSMALL)
            {
                perf->singular = 1;
                break;
            }
            const double alpha = wArA / wApA;
#pragma omp parallel for schedule(static) num_threads(nt) if (nt > 1)
            for (int32_t i = 0; i < n; ++i)
            {
                psi[i] += alpha * pA[i];
                rA[i] -= alpha * wA[i];
            }
            perf->finalResidual = sum_mag(n, rA, nt) / normFactor;
        } while ((++perf->nIterations < maxIter
                  && !orc_check_convergence(tolerance, relTol,
                                            perf->initialResidual,
                                            perf->finalResidual))
                 || perf->nIterations < minIter);
        free(P.rD);
    }
    perf->converged = orc_check_convergence(tolerance, relTol,
                                            perf->initialResidual,
                                            perf->finalResidual);
    free(pA);
    free(wA);
    free(rA);
    return 0;
}

int orc_foam_pbicgstab(int32_t n, int32_t nf, const int32_t* low,
                       const int32_t* upp, const int32_t* ownStart,
                       const int32_t* losort, const int32_t* losortStart,
                       const double* diag, const double* upper,
                       const double* lower, double* psi,
                       const double* source, double tolerance, double relTol,
                       int32_t maxIter, int32_t minIter, int32_t nthreads,
                       orc_foam_perf* perf)
{
    const int nt = nthreads > 1 ? nthreads : 1;
    memset(perf, 0, sizeof(*perf));
    if (!lower) lower = upper;
    const size_t nb = sizeof(double) * (size_t)(n > 0 ? n : 1);
    double* yA = (double*)malloc(nb);
    double* pA = (double*)malloc(nb);
    double* rA = (double*)malloc(nb);
    double* rA0 = (double*)malloc(nb);
    double* AyA = (double*)malloc(nb);
    double* sA = (double*)malloc(nb);
    double* zA = (double*)malloc(nb);
    double* tA = (double*)malloc(nb);
    double* rD = (double*)malloc(nb);

    orc_amul_rows(n, low, upp, ownStart, losort, losortStart, diag, upper,
                  lower, psi, yA, 0, nt);
    for (int32_t i = 0; i < n; ++i) rA[i] = source[i] - yA[i];
    orc_sumA(n, nf, low, upp, diag, upper, lower, pA);
    const double normFactor = orc_normfactor(n, psi, source, yA, pA);
    perf->initialResidual = sum_mag(n, rA, nt) / normFactor;
    perf->finalResidual = perf->initialResidual;

    if (minIter > 0
        || !orc_check_convergence(tolerance, relTol, perf->initialResidual,
                                  perf->finalResidual))
    {
        for (int32_t i = 0; i < n; ++i) rD[i] = 1.0 / diag[i];
        memcpy(rA0, rA, nb);
        double rA0rA = 0.0, rA0rAold, alpha = 0.0, omega = 0.0;
        do
        {
            rA0rAold = rA0rA;
            rA0rA = sum_prod(n, rA0, rA, nt);
            if (fabs(rA0rA) < VSMALL)
            {
                perf->singular = 1;
                break;
            }
            if (perf->nIterations == 0)
            {
                memcpy(pA, rA, nb);
            }
            else
            {
                if (fabs(omega) < VSMALL)
                {
                    perf->singular = 1;
                    break;
                }
                const double beta = (rA0rA / rA0rAold) * (alpha / omega);
#pragma omp parallel for schedule(static) num_threads(nt) if (nt > 1)
                for (int32_t i = 0; i < n; ++i)
                    pA[i] = rA[i] + beta * (pA[i] - omega * AyA[i]);
            }
#pragma omp parallel for schedule(static) num_threads(nt) if (nt > 1)
            for (int32_t i = 0; i < n; ++i) yA[i] = rD[i] * pA[i];
            orc_amul_rows(n, low, upp, ownStart, losort, losortStart, diag,
                          upper, lower, yA, AyA, 0, nt);
            const double rA0AyA = sum_prod(n, rA0, AyA, nt);
            alpha = rA0rA / rA0AyA;
#pragma omp parallel for schedule(static) num_threads(nt) if (nt > 1)
            for (int32_t i = 0; i < n; ++i) sA[i] = rA[i] - alpha * AyA[i];
            perf->finalResidual = sum_mag(n, sA, nt) / normFactor;
            if (perf->nIterations >= minIter
                && orc_check_convergence(tolerance, relTol,
                                         perf->initialResidual,
                                         perf->finalResidual))
            {
                for (int32_t i = 0; i < n; ++i) psi[i] += alpha * yA[i];
                perf->nIterations++;
                perf->converged = 1;
                goto done;
            }
#pragma omp parallel for schedule(static) num_threads(nt) if (nt > 1)
            for (int32_t i = 0; i < n; ++i) zA[i] = rD[i] * sA[i];
            orc_amul_rows(n, low, upp, ownStart, losort, losortStart, diag,
                          upper, lower, zA, tA, 0, nt);
            const double tAtA = sum_prod(n, tA, tA, nt);
            omega = sum_prod(n, tA, sA, nt) / tAtA;
#pragma omp parallel for schedule(static) num_threads(nt) if (nt > 1)
            for (int32_t i = 0; i < n; ++i)
            {
                psi[i] += alpha * yA[i] + omega * zA[i];
                rA[i] = sA[i] - omega * tA[i];
            }
            perf->finalResidual = sum_mag(n, rA, nt) / normFactor;
        } while ((++perf->nIterations < maxIter
                  && !orc_check_convergence(tolerance, relTol,
                                            perf->initialResidual,
                                            perf->finalResidual))
                 || perf->nIterations < minIter);
    }
    perf->converged = orc_check_convergence(tolerance, relTol,
                                            perf->initialResidual,
                                            perf->finalResidual);
done:
    free(yA);
    free(pA);
    free(rA);
    free(rA0);
    free(AyA);
    free(sA);
    free(zA);
    free(tA);
    free(rD);
    return 0;
}

static double norm2(int32_t n, const double* a, int nt)
{
    return sqrt(sum_prod(n, a, a, nt));
}

int orc_cg64(int32_t n, int32_t nf, const int32_t* low, const int32_t* upp,
             const int32_t* ownStart, const int32_t* losort,
             const int32_t* losortStart, const double* diag,
             const double* upper, const double* lower, double* x,
             const double* b, double tol_l2, int32_t maxIter,
             int32_t transpose, int32_t nthreads)
{
    (void)nf;
    const int nt = nthreads > 1 ? nthreads : 1;
    const size_t nb = sizeof(double) * (size_t)(n > 0 ? n : 1);
    double* r = (double*)malloc(nb);
    double* z = (double*)malloc(nb);
    double* p = (double*)malloc(nb);
    double* q = (double*)malloc(nb);
    double* rD = (double*)malloc(nb);
    int it = 0;
    const double bn = norm2(n, b, nt);
    const double stop = tol_l2 * (bn > 0 ? bn : 1.0);
    for (int32_t i = 0; i < n; ++i) rD[i] = 1.0 / diag[i];
    orc_amul_rows(n, low, upp, ownStart, losort, losortStart, diag, upper,
                  lower, x, q, transpose, nt);
    for (int32_t i = 0; i < n; ++i) r[i] = b[i] - q[i];
    if (!lower)
    {
        /* Deflated Jacobi-PCG (Nicolaides deflation with the constant vector,
         * Z = 1): pressure matrices with one pinned cell have a weakly held
         * constant mode, and right-hand sides with a large mean give
         * solutions with a large constant offset that plain CG resolves
         * slowly and only to offset-limited accuracy.  With u = A 1 and
         * sigma = 1.u: P = I - u 1^T/sigma, CG on P A xt = P b, and
         * x = 1 (1.b)/sigma + xt - 1 (u.xt)/sigma; the residual of x equals
         * P (b - A xt), the quantity iterated on.  Starts from x = 0. */
        double* u = (double*)malloc(nb);
        double* xt = (double*)malloc(nb);
        for (int32_t i = 0; i < n; ++i) z[i] = 1.0;
        orc_amul_rows(n, low, upp, ownStart, losort, losortStart, diag, upper, NULL, z, u,
                      transpose, nt);
        double sigma = 0.0;
        for (int32_t i = 0; i < n; ++i) sigma += u[i];
        const int defl = sigma > 0.0;
#define CF_PROJECT(v)                                          \
    do                                                         \
    {                                                          \
        if (defl)                                              \
        {                                                      \
            double s_ = 0.0;                                   \
            for (int32_t i = 0; i < n; ++i) s_ += (v)[i];      \
            const double c_ = s_ / sigma;                      \
            for (int32_t i = 0; i < n; ++i) (v)[i] -= c_ * u[i]; \
        }                                                      \
    } while (0)
        memset(xt, 0, nb);
        memcpy(r, b, nb);
        CF_PROJECT(r);
        double rz = 0.0, rzold;
        for (it = 0; it < maxIter; ++it)
        {
            if (norm2(n, r, nt) <= stop) break;
            for (int32_t i = 0; i < n; ++i) z[i] = rD[i] * r[i];
            rzold = rz;
            rz = sum_prod(n, r, z, nt);
            if (it == 0) memcpy(p, z, nb);
            else
            {
                const double beta = rz / rzold;
                for (int32_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
            }
            orc_amul_rows(n, low, upp, ownStart, losort, losortStart, diag,
                          upper, NULL, p, q, transpose, nt);
            CF_PROJECT(q);
            const double alpha = rz / sum_prod(n, p, q, nt);
            for (int32_t i = 0; i < n; ++i)
            {
                xt[i] += alpha * p[i];
                r[i] -= alpha * q[i];
            }
            if ((it + 1) % 50 == 0)
            {
                /* recompute the true (deflated) residual to stop FP64 drift */
                orc_amul_rows(n, low, upp, ownStart, losort, losortStart,
                              diag, upper, NULL, xt, q, transpose, nt);
                for (int32_t i = 0; i < n; ++i) r[i] = b[i] - q[i];
                CF_PROJECT(r);
            }
        }
#undef CF_PROJECT
        if (defl)
        {
            double sb = 0.0, ux = 0.0;
            for (int32_t i = 0; i < n; ++i)
            {
                sb += b[i];
                ux += u[i] * xt[i];
            }
            const double c = (sb - ux) / sigma;
            for (int32_t i = 0; i < n; ++i) x[i] = xt[i] + c;
        }
        else
        {
            memcpy(x, xt, nb);
        }
        free(u);
        free(xt);
    }
    else
    {
        /* Jacobi-preconditioned BiCGStab with periodic true residual */
        double* r0 = (double*)malloc(nb);
        double* s = (double*)malloc(nb);
        double* y = (double*)malloc(nb);
        double* t = (double*)malloc(nb);
        double* v = (double*)malloc(nb);
        memcpy(r0, r, nb);
        memset(p, 0, nb);
        memset(v, 0, nb);
        double rho = 1.0, alpha = 1.0, omega = 1.0;
        for (it = 0; it < maxIter; ++it)
        {
            if (norm2(n, r, nt) <= stop) break;
            const double rhoNew = sum_prod(n, r0, r, nt);
            const double beta = (rhoNew / rho) * (alpha / omega);
            rho = rhoNew;
            for (int32_t i = 0; i < n; ++i) p[i] = r[i] + beta * (p[i] - omega * v[i]);
            for (int32_t i = 0; i < n; ++i) y[i] = rD[i] * p[i];
            orc_amul_rows(n, low, upp, ownStart, losort, losortStart, diag,
                          upper, lower, y, v, transpose, nt);
            alpha = rho / sum_prod(n, r0, v, nt);
            for (int32_t i = 0; i < n; ++i) s[i] = r[i] - alpha * v[i];
            for (int32_t i = 0; i < n; ++i) z[i] = rD[i] * s[i];
            orc_amul_rows(n, low, upp, ownStart, losort, losortStart, diag,
                          upper, lower, z, t, transpose, nt);
            omega = sum_prod(n, t, s, nt) / sum_prod(n, t, t, nt);
            for (int32_t i = 0; i < n; ++i)
            {
                x[i] += alpha * y[i] + omega * z[i];
                r[i] = s[i] - omega * t[i];
            }
            if ((it + 1) % 50 == 0)
            {
                orc_amul_rows(n, low, upp, ownStart, losort, losortStart,
                              diag, upper, lower, x, q, transpose, nt);
                for (int32_t i = 0; i < n; ++i) r[i] = b[i] - q[i];
            }
        }
        free(r0);
        free(s);
        free(y);
        free(t);
        free(v);
    }
    free(r);
    free(z);
    free(p);
    free(q);
    free(rD);
    return it < maxIter ? it : -it;
}
