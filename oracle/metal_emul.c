/*
 * metal_emul.c -- the reference's own algorithm restated in C (test oracle).
 *
 *  - the 14 MSL kernels of src/metal4Foam/shaders/metalFoamKernels.metal,
 *    emulated in IEEE FP32 (compile with -ffp-contract=off so no product is
 *    fused into an add, as the source's separate * and + read);
 *  - the two-stage thread-group reduction tg_sum (metalFoamKernels.metal:34-52)
 *    with simd_sum as a 5-level xor butterfly over 32 lanes;
 *  - the backend's staging, Chebyshev constants and PCG / BiCGStab encode
 *    loops (src/metal4Foam/backend/metalFoamBackend.C:342-385, 522-959);
 *  - the FP64 refinement driver solveImpl
 *    (src/metal4Foam/solvers/metalFoamSolver.C:77-437).
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define TG 256
#define SIMD 32

enum
{
    S_WARA = 0, S_WARAOLD, S_WAPA, S_ALPHA, S_BETA, S_RES,
    S_RA0RA, S_RA0RAOLD, S_RA0AYA, S_OMEGA, S_TATA, S_TASA,
    S_COUNT = 16
};

/* simd_sum over one simd group: xor butterfly, every lane ends with the
 * same value, lane 0's is returned. */
static float simd_sum32(const float* v)
{
    float a[SIMD], b[SIMD];
    memcpy(a, v, sizeof(a));
    for (int off = SIMD / 2; off >= 1; off >>= 1)
    {
        for (int l = 0; l < SIMD; ++l) b[l] = a[l] + a[l ^ off];
        memcpy(a, b, sizeof(a));
    }
    return a[0];
}

/* tg_sum over one thread group of TG values (metalFoamKernels.metal:34-52) */
static float tg_sum256(const float* v)
{
    float sh[SIMD];
    const int nsg = TG / SIMD;
    for (int sg = 0; sg < nsg; ++sg) sh[sg] = simd_sum32(v + sg * SIMD);
    for (int l = nsg; l < SIMD; ++l) sh[l] = 0.0f;
    return simd_sum32(sh);
}

static int32_t ngroups_of(int32_t n) { return (n + TG - 1) / TG; }

/* Reduce per-thread values v[0..n) into one partial per thread group;
 * threads past n contribute 0. */
static void group_partials(int32_t n, const float* v, float* partials)
{
    float buf[TG];
    const int32_t g = ngroups_of(n);
    for (int32_t t = 0; t < g; ++t)
    {
        for (int l = 0; l < TG; ++l)
        {
            const int64_t gid = (int64_t)t * TG + l;
            buf[l] = gid < n ? v[gid] : 0.0f;
        }
        partials[t] = tg_sum256(buf);
    }
}

static float ldu_row(const orc_ldu32* A, const float* x, int32_t i)
{
    float sum = A->diag[i] * x[i];
    for (int32_t f = A->ownStart[i]; f < A->ownStart[i + 1]; ++f)
        sum += A->upper[f] * x[A->upp[f]];
    for (int32_t k = A->losortStart[i]; k < A->losortStart[i + 1]; ++k)
    {
        const int32_t f = A->losort[k];
        sum += A->lower[f] * x[A->low[f]];
    }
    return sum;
}

void orc_k_ldu_spmv_dotw(const orc_ldu32* A, const float* x, const float* w,
                         float* y, float* partials)
{
    float* dv = (float*)malloc(sizeof(float) * (size_t)(A->n > 0 ? A->n : 1));
    for (int32_t i = 0; i < A->n; ++i)
    {
        const float sum = ldu_row(A, x, i);
        y[i] = sum;
        dv[i] = w[i] * sum;
    }
    group_partials(A->n, dv, partials);
    free(dv);
}

void orc_k_ldu_spmv(const orc_ldu32* A, const float* x, float* y)
{
    for (int32_t i = 0; i < A->n; ++i) y[i] = ldu_row(A, x, i);
}

void orc_k_cheb_init(int32_t n, const float* r, const float* rD, float* w,
                     float* z, float c1)
{
    for (int32_t i = 0; i < n; ++i)
    {
        const float wi = c1 * rD[i] * r[i];
        w[i] = wi;
        z[i] = wi;
    }
}

void orc_k_cheb_step(int32_t n, const float* r, const float* v,
                     const float* rD, float* w, float* z, float c2, float c3)
{
    for (int32_t i = 0; i < n; ++i)
    {
        const float wi = c2 * w[i] + c3 * rD[i] * (r[i] - v[i]);
        w[i] = wi;
        z[i] += wi;
    }
}

void orc_k_emul(int32_t n, const float* a, const float* b, float* out)
{
    for (int32_t i = 0; i < n; ++i) out[i] = a[i] * b[i];
}

void orc_k_pcg_precond_dot(int32_t n, const float* rA, const float* rD,
                           float* wA, float* partials)
{
    float* dv = (float*)malloc(sizeof(float) * (size_t)(n > 0 ? n : 1));
    for (int32_t i = 0; i < n; ++i)
    {
        const float wv = rA[i] * rD[i];
        wA[i] = wv;
        dv[i] = wv * rA[i];
    }
    group_partials(n, dv, partials);
    free(dv);
}

void orc_k_pcg_update_p(int32_t n, float* p, const float* wA, const float* s)
{
    for (int32_t i = 0; i < n; ++i) p[i] = wA[i] + s[S_BETA] * p[i];
}

void orc_k_pcg_update_sol_res(int32_t n, float* delta, float* rA,
                              const float* p, const float* wA, const float* s,
                              float* partials)
{
    float* m = (float*)malloc(sizeof(float) * (size_t)(n > 0 ? n : 1));
    const float a = s[S_ALPHA];
    for (int32_t i = 0; i < n; ++i)
    {
        delta[i] += a * p[i];
        const float r = rA[i] - a * wA[i];
        rA[i] = r;
        m[i] = fabsf(r);
    }
    group_partials(n, m, partials);
    free(m);
}

void orc_k_dot_partial(int32_t n, const float* a, const float* b,
                       float* partials)
{
    float* v = (float*)malloc(sizeof(float) * (size_t)(n > 0 ? n : 1));
    for (int32_t i = 0; i < n; ++i) v[i] = a[i] * b[i];
    group_partials(n, v, partials);
    free(v);
}

void orc_k_reduce_scalars(const float* P1, const float* P2, float* s,
                          uint32_t count, uint32_t mode, uint32_t firstIter)
{
    float v1[TG], v2[TG];
    for (int l = 0; l < TG; ++l)
    {
        float a = 0.0f, b = 0.0f;
        for (uint32_t i = (uint32_t)l; i < count; i += TG)
        {
            a += P1[i];
            if (mode == 5) b += P2[i];
        }
        v1[l] = a;
        v2[l] = b;
    }
    const float t1 = tg_sum256(v1);
    const float t2 = (mode == 5) ? tg_sum256(v2) : 0.0f;
    switch (mode)
    {
        case 0:
            s[S_WARAOLD] = s[S_WARA];
            s[S_WARA] = t1;
            s[S_BETA] = firstIter ? 0.0f : t1 / s[S_WARAOLD];
            break;
        case 1:
            s[S_WAPA] = t1;
            s[S_ALPHA] = s[S_WARA] / t1;
            break;
        case 2:
            s[S_RES] = t1;
            break;
        case 3:
            s[S_RA0RAOLD] = s[S_RA0RA];
            s[S_RA0RA] = t1;
            s[S_BETA] = firstIter
                ? 0.0f
                : (t1 / s[S_RA0RAOLD]) * (s[S_ALPHA] / s[S_OMEGA]);
            break;
        case 4:
            s[S_RA0AYA] = t1;
            s[S_ALPHA] = s[S_RA0RA] / t1;
            break;
        case 5:
            s[S_TATA] = t1;
            s[S_TASA] = t2;
            s[S_OMEGA] = t2 / t1;
            break;
        default:
            break;
    }
}

void orc_k_bicg_update_p(int32_t n, float* p, const float* rA,
                         const float* AyA, const float* s)
{
    for (int32_t i = 0; i < n; ++i)
        p[i] = rA[i] + s[S_BETA] * (p[i] - s[S_OMEGA] * AyA[i]);
}

void orc_k_bicg_s_res(int32_t n, float* sA, const float* rA, const float* AyA,
                      const float* s, float* partials)
{
    float* m = (float*)malloc(sizeof(float) * (size_t)(n > 0 ? n : 1));
    for (int32_t i = 0; i < n; ++i)
    {
        const float sv = rA[i] - s[S_ALPHA] * AyA[i];
        sA[i] = sv;
        m[i] = fabsf(sv);
    }
    group_partials(n, m, partials);
    free(m);
}

void orc_k_bicg_early_update(int32_t n, float* delta, const float* yA,
                             const float* s)
{
    for (int32_t i = 0; i < n; ++i) delta[i] += s[S_ALPHA] * yA[i];
}

void orc_k_bicg_update_sol_res(int32_t n, float* delta, const float* yA,
                               const float* zA, float* rA, const float* sA,
                               const float* tA, const float* s,
                               float* partials)
{
    float* m = (float*)malloc(sizeof(float) * (size_t)(n > 0 ? n : 1));
    const float a = s[S_ALPHA];
    const float o = s[S_OMEGA];
    for (int32_t i = 0; i < n; ++i)
    {
        delta[i] += a * yA[i] + o * zA[i];
        const float r = sA[i] - o * tA[i];
        rA[i] = r;
        m[i] = fabsf(r);
    }
    group_partials(n, m, partials);
    free(m);
}

/* ------------------------------------------------------------- backend */

struct orc_backend
{
    int32_t n, nf, ngroups;
    const int32_t *low, *upp, *ownStart, *losort, *losortStart;
    float *diag, *upper, *lower, *rD;
    int32_t ownLower;
    float *rA, *p, *wA, *delta, *deltaBest, *chebW, *chebV;
    float *rA0, *yA, *AyA, *sA, *zA, *tA;
    float *P1, *P2, *P3;
    float s[S_COUNT];
};

static float* fzeros(int64_t n)
{
    return (float*)calloc((size_t)(n > 0 ? n : 1), sizeof(float));
}

orc_backend* orc_backend_new(int32_t n, int32_t nf, const int32_t* low,
                             const int32_t* upp, const int32_t* ownStart,
                             const int32_t* losort,
                             const int32_t* losortStart)
{
    orc_backend* b = (orc_backend*)calloc(1, sizeof(orc_backend));
    b->n = n;
    b->nf = nf;
    b->ngroups = ngroups_of(n);
    b->low = low;
    b->upp = upp;
    b->ownStart = ownStart;
    b->losort = losort;
    b->losortStart = losortStart;
    b->diag = fzeros(n);
    b->upper = fzeros(nf);
    b->lower = b->upper;
    b->rD = fzeros(n);
    b->rA = fzeros(n);
    b->p = fzeros(n);
    b->wA = fzeros(n);
    b->delta = fzeros(n);
    b->deltaBest = fzeros(n);
    b->chebW = fzeros(n);
    b->chebV = fzeros(n);
    b->rA0 = fzeros(n);
    b->yA = fzeros(n);
    b->AyA = fzeros(n);
    b->sA = fzeros(n);
    b->zA = fzeros(n);
    b->tA = fzeros(n);
    b->P1 = fzeros(b->ngroups);
    b->P2 = fzeros(b->ngroups);
    b->P3 = fzeros(b->ngroups);
    return b;
}

void orc_backend_free(orc_backend* b)
{
    if (!b) return;
    if (b->ownLower) free(b->lower);
    float* arrs[] = {b->diag, b->upper, b->rD, b->rA, b->p, b->wA, b->delta,
                     b->deltaBest, b->chebW, b->chebV, b->rA0, b->yA, b->AyA,
                     b->sA, b->zA, b->tA, b->P1, b->P2, b->P3};
    for (size_t i = 0; i < sizeof(arrs) / sizeof(arrs[0]); ++i) free(arrs[i]);
    free(b);
}

void orc_backend_set_coeffs(orc_backend* b, const double* diag,
                            const double* upper, const double* lower)
{
    for (int32_t i = 0; i < b->n; ++i) b->diag[i] = (float)diag[i];
    for (int32_t f = 0; f < b->nf; ++f) b->upper[f] = (float)upper[f];
    if (lower)
    {
        if (!b->ownLower)
        {
            b->lower = fzeros(b->nf);
            b->ownLower = 1;
        }
        for (int32_t f = 0; f < b->nf; ++f) b->lower[f] = (float)lower[f];
    }
    else
    {
        if (b->ownLower) free(b->lower);
        b->ownLower = 0;
        b->lower = b->upper;
    }
    for (int32_t i = 0; i < b->n; ++i) b->rD[i] = (float)(1.0 / diag[i]);
}

const float* orc_backend_delta(const orc_backend* b) { return b->delta; }

static orc_ldu32 ldu_of(const orc_backend* b)
{
    orc_ldu32 A;
    A.n = b->n;
    A.nf = b->nf;
    A.diag = b->diag;
    A.upper = b->upper;
    A.lower = b->lower;
    A.low = b->low;
    A.upp = b->upp;
    A.ownStart = b->ownStart;
    A.losort = b->losort;
    A.losortStart = b->losortStart;
    return A;
}

void orc_cheb_constants(int32_t order, double beta, double ratio, float* c)
{
    const double alpha = beta / ratio;
    const double theta = 0.5 * (beta + alpha);
    const double delta = 0.5 * (beta - alpha);
    const double sigma = theta / delta;
    double rho = 1.0 / sigma;
    c[0] = (float)(1.0 / theta);
    for (int32_t i = 1; i < order; ++i)
    {
        const double rhoNew = 1.0 / (2.0 * sigma - rho);
        c[2 * i - 1] = (float)(rhoNew * rho);
        c[2 * i] = (float)(2.0 * rhoNew / delta);
        rho = rhoNew;
    }
}

static void enc_cheb(orc_backend* b, const orc_ldu32* A, const float* r,
                     float* z, int32_t order, const float* c)
{
    orc_k_cheb_init(b->n, r, b->rD, b->chebW, z, c[0]);
    for (int32_t i = 1; i < order; ++i)
    {
        orc_k_ldu_spmv(A, z, b->chebV);
        orc_k_cheb_step(b->n, r, b->chebV, b->rD, b->chebW, z, c[2 * i - 1],
                        c[2 * i]);
    }
}

orc_stats orc_backend_pcg(orc_backend* b, const double* r, double target,
                          int32_t maxIter, int32_t iterationsPerSync,
                          int32_t chebOrder, double chebBeta, double chebRatio)
{
    orc_stats st;
    memset(&st, 0, sizeof(st));
    const int32_t n = b->n;
    if (n == 0)
    {
        st.singular = 1;
        return st;
    }
    orc_ldu32 A = ldu_of(b);
    float* cc = NULL;
    if (chebOrder > 1)
    {
        cc = (float*)malloc(sizeof(float) * (size_t)(2 * chebOrder));
        orc_cheb_constants(chebOrder, chebBeta, chebRatio, cc);
    }
    for (int32_t i = 0; i < n; ++i) b->rA[i] = (float)r[i];
    memset(b->delta, 0, sizeof(float) * (size_t)n);
    memset(b->deltaBest, 0, sizeof(float) * (size_t)n);
    memset(b->p, 0, sizeof(float) * (size_t)n);
    memset(b->s, 0, sizeof(b->s));
    if (iterationsPerSync < 1) iterationsPerSync = 1;

    int32_t it = 0;
    double bestRes = 1.0e300;
    int32_t noProgress = 0;
    const int32_t stagLimit = 50;
    while (it < maxIter)
    {
        const int32_t batch = iterationsPerSync < maxIter - it
                                  ? iterationsPerSync : maxIter - it;
        for (int32_t k = 0; k < batch; ++k)
        {
            const uint32_t firstIter = (it + k == 0) ? 1u : 0u;
            if (chebOrder > 1)
            {
                enc_cheb(b, &A, b->rA, b->wA, chebOrder, cc);
                orc_k_dot_partial(n, b->wA, b->rA, b->P1);
            }
            else
            {
                orc_k_pcg_precond_dot(n, b->rA, b->rD, b->wA, b->P1);
            }
            orc_k_reduce_scalars(b->P1, b->P1, b->s, (uint32_t)b->ngroups, 0,
                                 firstIter);
            orc_k_pcg_update_p(n, b->p, b->wA, b->s);
            orc_k_ldu_spmv_dotw(&A, b->p, b->p, b->wA, b->P2);
            orc_k_reduce_scalars(b->P2, b->P2, b->s, (uint32_t)b->ngroups, 1, 0);
            orc_k_pcg_update_sol_res(n, b->delta, b->rA, b->p, b->wA, b->s,
                                     b->P3);
            orc_k_reduce_scalars(b->P3, b->P3, b->s, (uint32_t)b->ngroups, 2, 0);
        }
        it += batch;
        st.nIterations = it;
        const double res = (double)b->s[S_RES];
        st.finalResSum = res;
        if (!isfinite(res) || !isfinite((double)b->s[S_WAPA]))
        {
            st.singular = 1;
            break;
        }
        if (res < bestRes)
        {
            bestRes = res;
            noProgress = 0;
            memcpy(b->deltaBest, b->delta, sizeof(float) * (size_t)n);
        }
        else
        {
            noProgress += batch;
        }
        if (res <= target)
        {
            st.converged = 1;
            break;
        }
        if (noProgress >= stagLimit)
        {
            st.stagnated = 1;
            break;
        }
    }
    if (bestRes < st.finalResSum)
    {
        memcpy(b->delta, b->deltaBest, sizeof(float) * (size_t)n);
        st.finalResSum = bestRes;
    }
    free(cc);
    return st;
}

orc_stats orc_backend_bicgstab(orc_backend* b, const double* r, double target,
                               int32_t maxIter)
{
    orc_stats st;
    memset(&st, 0, sizeof(st));
    const int32_t n = b->n;
    if (n == 0)
    {
        st.singular = 1;
        return st;
    }
    orc_ldu32 A = ldu_of(b);
    for (int32_t i = 0; i < n; ++i) b->rA[i] = (float)r[i];
    memcpy(b->rA0, b->rA, sizeof(float) * (size_t)n);
    memset(b->delta, 0, sizeof(float) * (size_t)n);
    memset(b->deltaBest, 0, sizeof(float) * (size_t)n);
    memset(b->p, 0, sizeof(float) * (size_t)n);
    memset(b->AyA, 0, sizeof(float) * (size_t)n);
    memset(b->s, 0, sizeof(b->s));
    const uint32_t ng = (uint32_t)b->ngroups;

    int32_t it = 0;
    double bestRes = 1.0e300;
    int32_t noProgress = 0;
    const int32_t stagLimit = 50;
    while (it < maxIter)
    {
        const uint32_t firstIter = (it == 0) ? 1u : 0u;
        orc_k_dot_partial(n, b->rA0, b->rA, b->P1);
        orc_k_reduce_scalars(b->P1, b->P1, b->s, ng, 3, firstIter);
        orc_k_bicg_update_p(n, b->p, b->rA, b->AyA, b->s);
        orc_k_emul(n, b->rD, b->p, b->yA);
        orc_k_ldu_spmv_dotw(&A, b->yA, b->rA0, b->AyA, b->P2);
        orc_k_reduce_scalars(b->P2, b->P2, b->s, ng, 4, 0);
        orc_k_bicg_s_res(n, b->sA, b->rA, b->AyA, b->s, b->P3);
        orc_k_reduce_scalars(b->P3, b->P3, b->s, ng, 2, 0);

        if (!isfinite((double)b->s[S_RA0RA]) || !isfinite((double)b->s[S_ALPHA])
            || !isfinite((double)b->s[S_RES]))
        {
            st.singular = 1;
            break;
        }
        {
            const double res = (double)b->s[S_RES];
            if (res <= target)
            {
                orc_k_bicg_early_update(n, b->delta, b->yA, b->s);
                st.nIterations = ++it;
                st.finalResSum = res;
                st.converged = 1;
                return st;
            }
        }
        orc_k_emul(n, b->rD, b->sA, b->zA);
        orc_k_ldu_spmv_dotw(&A, b->zA, b->sA, b->tA, b->P2);
        orc_k_dot_partial(n, b->tA, b->tA, b->P1);
        orc_k_reduce_scalars(b->P1, b->P2, b->s, ng, 5, 0);
        orc_k_bicg_update_sol_res(n, b->delta, b->yA, b->zA, b->rA, b->sA,
                                  b->tA, b->s, b->P3);
        orc_k_reduce_scalars(b->P3, b->P3, b->s, ng, 2, 0);

        ++it;
        st.nIterations = it;
        const double res = (double)b->s[S_RES];
        st.finalResSum = res;
        if (!isfinite(res) || !isfinite((double)b->s[S_OMEGA]))
        {
            st.singular = 1;
            break;
        }
        if (res < bestRes)
        {
            bestRes = res;
            noProgress = 0;
            memcpy(b->deltaBest, b->delta, sizeof(float) * (size_t)n);
        }
        else
        {
            noProgress += 1;
        }
        if (res <= target)
        {
            st.converged = 1;
            break;
        }
        if (noProgress >= stagLimit)
        {
            st.stagnated = 1;
            break;
        }
    }
    if (bestRes < st.finalResSum)
    {
        memcpy(b->delta, b->deltaBest, sizeof(float) * (size_t)n);
        st.finalResSum = bestRes;
    }
    return st;
}

/* ------------------------------------------------------------- driver */

#define VSMALL 1.0e-300

int orc_metal_solve(int32_t n, int32_t nf, const int32_t* low,
                    const int32_t* upp, const int32_t* ownStart,
                    const int32_t* losort, const int32_t* losortStart,
                    const double* diag, const double* upper,
                    const double* lower, double* psi, const double* source,
                    int32_t useBiCGStab, const orc_controls* ctl,
                    orc_perf* perf)
{
    memset(perf, 0, sizeof(*perf));
    const size_t nb = sizeof(double) * (size_t)(n > 0 ? n : 1);
    double* wA = (double*)malloc(nb);
    double* rA = (double*)malloc(nb);
    double* u = (double*)malloc(nb);
    double* diag0 = (double*)malloc(nb);
    double* rin = (double*)malloc(nb);
    double* sumOff = (double*)malloc(nb);

    /* initial FP64 residual and normalisation (metalFoamSolver.C:109-129) */
    orc_amul(n, nf, low, upp, diag, upper, lower, psi, wA);
    for (int32_t i = 0; i < n; ++i) rA[i] = source[i] - wA[i];
    orc_sumA(n, nf, low, upp, diag, upper, lower, u);
    const double normFactor = orc_normfactor(n, psi, source, wA, u);
    perf->normFactor = normFactor;
    perf->initialResidual = orc_sum_mag(n, rA) / normFactor;
    perf->finalResidual = perf->initialResidual;

    if (ctl->minIter > 0
        || !orc_check_convergence(ctl->tolerance, ctl->relTol,
                                  perf->initialResidual, perf->finalResidual))
    {
        perf->solved = 1;
        orc_backend* bk = orc_backend_new(n, nf, low, upp, ownStart, losort,
                                          losortStart);
        /* deflation decision (metalFoamSolver.C:167-209) */
        int deflate = 0;
        if (!useBiCGStab && ctl->deflate != 2)
        {
            if (ctl->deflate == 1)
            {
                deflate = 1;
            }
            else
            {
                int64_t nPinned = 0;
                for (int32_t i = 0; i < n; ++i)
                    if (fabs(u[i]) > 1e-8 * fabs(diag[i])) ++nPinned;
                deflate = (10 * nPinned <= (int64_t)n);
            }
        }
        const double* diagPtr = diag;
        if (deflate)
        {
            for (int32_t i = 0; i < n; ++i)
            {
                diag0[i] = diag[i] - u[i];
                if (diag0[i] * diag[i] <= VSMALL * fabs(diag0[i]))
                {
                    deflate = 0;
                    break;
                }
            }
            if (deflate) diagPtr = diag0;
        }
        perf->deflated = deflate;
        orc_backend_set_coeffs(bk, diagPtr, upper,
                               (!useBiCGStab || !lower) ? NULL : lower);

        /* Chebyshev setup, Gershgorin bound (metalFoamSolver.C:224-249) */
        const int32_t chebOrder = useBiCGStab ? 1 : ctl->chebyshevOrder;
        const double chebRatio = ctl->chebyshevRatio;
        double chebBeta = 2.0;
        if (chebOrder > 1)
        {
            for (int32_t i = 0; i < n; ++i) sumOff[i] = 0.0;
            for (int32_t f = 0; f < nf; ++f)
            {
                sumOff[low[f]] += fabs(upper[f]);
                sumOff[upp[f]] += fabs(upper[f]);
            }
            chebBeta = 0.0;
            for (int32_t i = 0; i < n; ++i)
            {
                const double g = 1.0 + sumOff[i] / fabs(diagPtr[i]);
                if (g > chebBeta) chebBeta = g;
            }
        }
        perf->chebBeta = chebBeta;

        const double tgt =
            (ctl->tolerance > ctl->relTol * perf->initialResidual
                 ? ctl->tolerance : ctl->relTol * perf->initialResidual)
            * normFactor;
        int32_t totalIter = 0;
        int32_t outer;
        int singular = 0;
        double prevRes = perf->initialResidual;

        for (outer = 0; outer <= ctl->maxRestarts; ++outer)
        {
            const double* rPtr = rA;
            if (deflate)
            {
                double mean = 0.0;
                for (int32_t i = 0; i < n; ++i) mean += rA[i];
                mean /= n;
                for (int32_t i = 0; i < n; ++i) rin[i] = rA[i] - mean;
                rPtr = rin;
            }
            orc_stats st = useBiCGStab
                ? orc_backend_bicgstab(bk, rPtr, tgt, ctl->maxIter - totalIter)
                : orc_backend_pcg(bk, rPtr, tgt, ctl->maxIter - totalIter,
                                  ctl->iterationsPerSync, chebOrder, chebBeta,
                                  chebRatio);
            totalIter += st.nIterations;
            singular = st.singular;

            const float* del = orc_backend_delta(bk);
            double delMean = 0.0;
            if (deflate)
            {
                for (int32_t i = 0; i < n; ++i) delMean += del[i];
                delMean /= n;
            }
            for (int32_t i = 0; i < n; ++i) psi[i] += (double)del[i] - delMean;

            orc_amul(n, nf, low, upp, diag, upper, lower, psi, wA);
            for (int32_t i = 0; i < n; ++i) rA[i] = source[i] - wA[i];

            if (deflate)
            {
                double ur = 0.0, uu = 0.0;
                for (int32_t i = 0; i < n; ++i)
                {
                    ur += u[i] * rA[i];
                    uu += u[i] * u[i];
                }
                if (uu > VSMALL)
                {
                    const double c = ur / uu;
                    for (int32_t i = 0; i < n; ++i)
                    {
                        psi[i] += c;
                        rA[i] -= c * u[i];
                    }
                }
            }
            perf->finalResidual = orc_sum_mag(n, rA) / normFactor;
            perf->nIterations = totalIter;

            if (deflate && perf->finalResidual > prevRes / 1.5 && !st.singular)
            {
                deflate = 0;
                perf->polished = 1;
                orc_backend_set_coeffs(bk, diag, upper, NULL);
            }
            prevRes = perf->finalResidual;

            if (singular) break;
            if (totalIter >= ctl->maxIter) break;
            if (perf->nIterations >= ctl->minIter
                && orc_check_convergence(ctl->tolerance, ctl->relTol,
                                         perf->initialResidual,
                                         perf->finalResidual))
                break;
        }
        perf->nRestarts = outer;
        perf->singular = singular;
        orc_backend_free(bk);
    }
    perf->converged = orc_check_convergence(ctl->tolerance, ctl->relTol,
                                            perf->initialResidual,
                                            perf->finalResidual);
    free(wA);
    free(rA);
    free(u);
    free(diag0);
    free(rin);
    free(sumOff);
    return 0;
}
