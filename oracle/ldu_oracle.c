/*
 * ldu_oracle.c -- OpenFOAM v2506 LDU semantics the reference driver calls
 * (metalFoamSolver.C:109,120,128,134,152-158,168,333,364,410), restated in
 * plain C as the test oracle.  OpenFOAM is a third-party dependency that is
 * not vendored with the reference; the functions follow its documented
 * behaviour and are pinned here only by hand-checked known-answer tests.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

int orc_build_addressing(int32_t n, int32_t nf, const int32_t* low,
                         const int32_t* upp, int32_t* ownStart,
                         int32_t* losort, int32_t* losortStart)
{
    if (n < 0 || nf < 0) return -1;
    for (int32_t f = 0; f < nf; ++f)
    {
        if (low[f] < 0 || upp[f] >= n || low[f] >= upp[f]) return -1;
        if (f > 0)
        {
            if (low[f] < low[f - 1]) return -1;
            if (low[f] == low[f - 1] && upp[f] <= upp[f - 1]) return -1;
        }
    }
    /* ownerStart: counting sort of owners (faces are owner-sorted) */
    memset(ownStart, 0, sizeof(int32_t) * (size_t)(n + 1));
    for (int32_t f = 0; f < nf; ++f) ownStart[low[f] + 1]++;
    for (int32_t i = 0; i < n; ++i) ownStart[i + 1] += ownStart[i];
    /* losort: stable counting sort of faces by neighbour */
    memset(losortStart, 0, sizeof(int32_t) * (size_t)(n + 1));
    for (int32_t f = 0; f < nf; ++f) losortStart[upp[f] + 1]++;
    for (int32_t i = 0; i < n; ++i) losortStart[i + 1] += losortStart[i];
    int32_t* fill = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    if (!fill) return -1;
    memcpy(fill, losortStart, sizeof(int32_t) * (size_t)n);
    for (int32_t f = 0; f < nf; ++f) losort[fill[upp[f]]++] = f;
    free(fill);
    return 0;
}

static void amul_impl(int32_t n, int32_t nf, const int32_t* low,
                      const int32_t* upp, const double* diag,
                      const double* upper, const double* lower,
                      const double* x, double* y)
{
    if (!lower) lower = upper;
    for (int32_t c = 0; c < n; ++c) y[c] = diag[c] * x[c];
    for (int32_t f = 0; f < nf; ++f)
    {
        y[upp[f]] += lower[f] * x[low[f]];
        y[low[f]] += upper[f] * x[upp[f]];
    }
}

void orc_amul(int32_t n, int32_t nf, const int32_t* low, const int32_t* upp,
              const double* diag, const double* upper, const double* lower,
              const double* x, double* y)
{
    amul_impl(n, nf, low, upp, diag, upper, lower, x, y);
}

void orc_tmul(int32_t n, int32_t nf, const int32_t* low, const int32_t* upp,
              const double* diag, const double* upper, const double* lower,
              const double* x, double* y)
{
    /* lduMatrix::Tmul: the same loop with upper and lower exchanged */
    amul_impl(n, nf, low, upp, diag, lower ? lower : upper, upper, x, y);
}

void orc_sumA(int32_t n, int32_t nf, const int32_t* low, const int32_t* upp,
              const double* diag, const double* upper, const double* lower,
              double* u)
{
    if (!lower) lower = upper;
    for (int32_t c = 0; c < n; ++c) u[c] = diag[c];
    for (int32_t f = 0; f < nf; ++f)
    {
        u[upp[f]] += lower[f];
        u[low[f]] += upper[f];
    }
}

double orc_normfactor(int32_t n, const double* psi, const double* source,
                      const double* Apsi, const double* sumA)
{
    double xRef = 0.0;
    for (int32_t i = 0; i < n; ++i) xRef += psi[i];
    xRef /= (double)(n > 0 ? n : 1);
    double s = 0.0;
    for (int32_t i = 0; i < n; ++i)
    {
        const double pA = sumA[i] * xRef;
        s += fabs(Apsi[i] - pA) + fabs(source[i] - pA);
    }
    return s + 1e-20;
}

double orc_sum_mag(int32_t n, const double* r)
{
    double s = 0.0;
    for (int32_t i = 0; i < n; ++i) s += fabs(r[i]);
    return s;
}

int orc_check_convergence(double tol, double relTol, double initial,
                          double final_)
{
    return (final_ < tol) || (relTol > 1e-20 && final_ < relTol * initial);
}

void orc_face_gradients(int32_t n, int32_t nf, const int32_t* low,
                        const int32_t* upp, const double* lambda,
                        const double* x, double* dUpper, double* dLower,
                        double* dDiag)
{
    for (int32_t f = 0; f < nf; ++f)
    {
        dUpper[f] = -lambda[low[f]] * x[upp[f]];
        dLower[f] = -lambda[upp[f]] * x[low[f]];
    }
    for (int32_t i = 0; i < n; ++i) dDiag[i] = -lambda[i] * x[i];
}
