/*
 * A C caller of libcudafoam: builds the LDU addressing of an nx x ny x nz
 * 7-point Poisson problem (faces in upper-triangular order, ownerStart,
 * losort, losortStart), fixes cell 0 (diag doubled, as OpenFOAM's
 * setReference), and solves it with cf_solve (cudaPCG) to 1e-6.
 *
 *   solve_poisson nx ny nz [GAMG]
 *
 * With GAMG the inner PCG is preconditioned by the multigrid V-cycle
 * (cf_options.preconditioner = CF_PRECOND_GAMG) instead of Chebyshev-Jacobi.
 * Prints "status <code>" and, on success, the solverPerformance figures and
 * the FP64 residual recomputed here from psi.  Exits 0 on CF_OK, 3 when no
 * sm_100 device is present (CF_ERR_NO_DEVICE), 1 otherwise.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "cudafoam.h"

static int idx(int i, int j, int k, int nx, int ny) { return i + nx * (j + ny * k); }

int main(int argc, char** argv)
{
    const int nx = argc > 1 ? atoi(argv[1]) : 24;
    const int ny = argc > 2 ? atoi(argv[2]) : 20;
    const int nz = argc > 3 ? atoi(argv[3]) : 16;
    const int n = nx * ny * nz;
    int nf = 0;
    int32_t* low = malloc(sizeof(int32_t) * 3 * n);
    int32_t* upp = malloc(sizeof(int32_t) * 3 * n);
    /* faces sorted by owner, then neighbour: for each cell its +x, +y, +z neighbours */
    for (int c = 0; c < n; ++c)
    {
        const int i = c % nx, j = (c / nx) % ny, k = c / (nx * ny);
        if (i + 1 < nx) { low[nf] = c; upp[nf] = idx(i + 1, j, k, nx, ny); ++nf; }
        if (j + 1 < ny) { low[nf] = c; upp[nf] = idx(i, j + 1, k, nx, ny); ++nf; }
        if (k + 1 < nz) { low[nf] = c; upp[nf] = idx(i, j, k + 1, nx, ny); ++nf; }
    }
    int32_t* own = calloc(n + 1, sizeof(int32_t));
    int32_t* losS = calloc(n + 1, sizeof(int32_t));
    int32_t* los = malloc(sizeof(int32_t) * (nf > 0 ? nf : 1));
    for (int f = 0; f < nf; ++f) { own[low[f] + 1]++; losS[upp[f] + 1]++; }
    for (int c = 0; c < n; ++c) { own[c + 1] += own[c]; losS[c + 1] += losS[c]; }
    int32_t* pos = malloc(sizeof(int32_t) * n);
    for (int c = 0; c < n; ++c) pos[c] = losS[c];
    for (int f = 0; f < nf; ++f) los[pos[upp[f]]++] = f;   /* stable in f */

    double* diag = calloc(n, sizeof(double));
    double* upper = malloc(sizeof(double) * (nf > 0 ? nf : 1));
    double* src = malloc(sizeof(double) * n);
    double* psi = calloc(n, sizeof(double));
    for (int f = 0; f < nf; ++f) { upper[f] = -1.0; diag[low[f]] += 1.0; diag[upp[f]] += 1.0; }
    diag[0] *= 2.0;
    double mean = 0.0;
    for (int c = 0; c < n; ++c) { src[c] = sin(0.37 * c) + 0.25 * cos(1.3 * c); mean += src[c]; }
    for (int c = 0; c < n; ++c) src[c] -= mean / n;

    cf_context* ctx = NULL;
    int rc = cf_context_create(&ctx, 0);
    if (rc != CF_OK)
    {
        printf("status %d %s\n", rc, cf_last_error());
        return rc == CF_ERR_NO_DEVICE ? 3 : 1;
    }
    rc = cf_set_topology(ctx, n, nf, low, upp, own, los, losS);
    if (rc == CF_OK) rc = cf_set_coeffs(ctx, diag, upper, NULL, NULL);
    cf_options o;
    cf_options_default(&o);
    if (argc > 4 && strcmp(argv[4], "GAMG") == 0) o.preconditioner = CF_PRECOND_GAMG;
    cf_performance perf;
    if (rc == CF_OK) rc = cf_solve(ctx, CF_SOLVER_PCG, psi, src, &o, &perf);
    printf("status %d %s\n", rc, rc == CF_OK ? "" : cf_last_error());
    if (rc == CF_OK)
    {
        /* residual b - A psi in FP64 (row order of lduMatrix::Amul) */
        double* r = malloc(sizeof(double) * n);
        for (int c = 0; c < n; ++c) r[c] = src[c] - diag[c] * psi[c];
        for (int f = 0; f < nf; ++f)
        {
            r[upp[f]] += psi[low[f]];     /* -(lower * psi[l]) with lower = -1 */
            r[low[f]] += psi[upp[f]];
        }
        double l1 = 0.0;
        for (int c = 0; c < n; ++c) l1 += fabs(r[c]);
        printf("initial %.6e final %.6e iterations %d converged %d l1 %.6e normFactor %.6e\n",
               perf.initialResidual, perf.finalResidual, perf.nIterations, perf.converged, l1,
               perf.normFactor);
        free(r);
    }
    cf_context_destroy(ctx);
    free(low); free(upp); free(own); free(losS); free(los); free(pos);
    free(diag); free(upper); free(src); free(psi);
    return rc == CF_OK ? 0 : 1;
}
