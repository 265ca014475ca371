/*
 * oracle.h -- CPU restatement of the metal4Foam Krylov path (TEST
 * INFRASTRUCTURE ONLY: the parity tests, the smoke check and the bench's
 * CPU-baseline leg call it as the checker; the product never links it).
 *
 * Three groups of functions:
 *
 *  1. OpenFOAM v2506 FP64 semantics the reference calls into (third party,
 *     not vendored; restated from their documented behaviour, see the
 *     citations per function): lduAddressing, Amul, sumA, normFactor,
 *     gSumMag, checkConvergence.
 *  2. The reference's own algorithm: the 14 MSL kernels
 *     (src/metal4Foam/shaders/metalFoamKernels.metal) emulated in IEEE FP32
 *     with the same two-stage reduction tree, the backend encode loops
 *     (src/metal4Foam/backend/metalFoamBackend.C:342-385, 568-959) and the
 *     FP64 refinement driver (src/metal4Foam/solvers/metalFoamSolver.C:77-437).
 *  3. The reference's CPU path that the plugin mirrors (OpenFOAM's FP64 PCG
 *     and PBiCGStab loops, with diagonal / DIC preconditioning), an FP64 CG
 *     converged to a tight L2 tolerance, and the FP64 adjoint of a solve.
 *
 * Parity status: group 2's kernel arithmetic is pinned against the
 * reference's own kernel source compiled on the CPU (oracle/_ref, built by
 * oracle/Makefile from the reference's .metal file with a SIMT shim);
 * groups 1 and 3 restate third-party code that is absent here and are
 * pinned only by hand-checked known-answer tests (parity unpinned at the
 * OpenFOAM boundary).
 */
#ifndef CUDAFOAM_ORACLE_H
#define CUDAFOAM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- group 1 */

/* lduAddressing: ownerStart / losort / losortStart from owner/neighbour
 * arrays by counting sort.  Returns 0, or -1 if the faces are not in
 * upper-triangular LDU order (owner < neighbour, sorted by owner then
 * neighbour) or out of range. */
int orc_build_addressing(int32_t n, int32_t nf, const int32_t* low,
                         const int32_t* upp, int32_t* ownStart,
                         int32_t* losort, int32_t* losortStart);

/* y = A x, FP64, in the summation order of lduMatrix::Amul (diag, then the
 * faces in index order, which per row is: neighbour-side terms in losort
 * order, then owner-side terms).  lower == NULL: symmetric. */
void orc_amul(int32_t n, int32_t nf, const int32_t* low, const int32_t* upp,
              const double* diag, const double* upper, const double* lower,
              const double* x, double* y);

/* Same as orc_amul but the transpose (upper and lower swapped). */
void orc_tmul(int32_t n, int32_t nf, const int32_t* low, const int32_t* upp,
              const double* diag, const double* upper, const double* lower,
              const double* x, double* y);

/* u = A 1 (lduMatrix::sumA without interfaces). */
void orc_sumA(int32_t n, int32_t nf, const int32_t* low, const int32_t* upp,
              const double* diag, const double* upper, const double* lower,
              double* u);

/* lduMatrix::solver::normFactor (L1_SCALED): with xRef = mean(psi) and
 * pA = xRef*sumA, returns sum(|Apsi - pA| + |source - pA|) + 1e-20. */
double orc_normfactor(int32_t n, const double* psi, const double* source,
                      const double* Apsi, const double* sumA);

double orc_sum_mag(int32_t n, const double* r);

/* SolverPerformance::checkConvergence: final < tol, or relTol > 1e-20 and
 * final < relTol*initial. */
int orc_check_convergence(double tol, double relTol, double initial,
                          double final_);

/* ---------------------------------------------------------------- group 2 */

/* The FP32 emulation of every reference kernel, thread group 256, simd
 * group 32, simd_sum as a 5-level xor butterfly, one float partial per
 * thread group.  Buffers as in the MSL signatures. */
typedef struct
{
    int32_t n, nf;
    const float* diag;
    const float* upper;
    const float* lower;
    const int32_t* low;
    const int32_t* upp;
    const int32_t* ownStart;
    const int32_t* losort;
    const int32_t* losortStart;
} orc_ldu32;

void orc_k_ldu_spmv_dotw(const orc_ldu32* A, const float* x, const float* w,
                         float* y, float* partials);
void orc_k_ldu_spmv(const orc_ldu32* A, const float* x, float* y);
void orc_k_cheb_init(int32_t n, const float* r, const float* rD, float* w,
                     float* z, float c1);
void orc_k_cheb_step(int32_t n, const float* r, const float* v,
                     const float* rD, float* w, float* z, float c2, float c3);
void orc_k_emul(int32_t n, const float* a, const float* b, float* out);
void orc_k_pcg_precond_dot(int32_t n, const float* rA, const float* rD,
                           float* wA, float* partials);
void orc_k_pcg_update_p(int32_t n, float* p, const float* wA, const float* s);
void orc_k_pcg_update_sol_res(int32_t n, float* delta, float* rA,
                              const float* p, const float* wA, const float* s,
                              float* partials);
void orc_k_dot_partial(int32_t n, const float* a, const float* b,
                       float* partials);
void orc_k_reduce_scalars(const float* P1, const float* P2, float* s,
                          uint32_t count, uint32_t mode, uint32_t firstIter);
void orc_k_bicg_update_p(int32_t n, float* p, const float* rA,
                         const float* AyA, const float* s);
void orc_k_bicg_s_res(int32_t n, float* sA, const float* rA, const float* AyA,
                      const float* s, float* partials);
void orc_k_bicg_early_update(int32_t n, float* delta, const float* yA,
                             const float* s);
void orc_k_bicg_update_sol_res(int32_t n, float* delta, const float* yA,
                               const float* zA, float* rA, const float* sA,
                               const float* tA, const float* s,
                               float* partials);

/* metalFoamBackend::Stats (metalFoamBackend.H:41-50) */
typedef struct
{
    int32_t nIterations;
    double finalResSum;
    int32_t converged;
    int32_t singular;
    int32_t stagnated;
} orc_stats;

/* An emulated backend: FP32 copies of the coefficients plus work vectors. */
typedef struct orc_backend orc_backend;

orc_backend* orc_backend_new(int32_t n, int32_t nf, const int32_t* low,
                             const int32_t* upp, const int32_t* ownStart,
                             const int32_t* losort,
                             const int32_t* losortStart);
void orc_backend_free(orc_backend* b);
/* metalFoamBackend::setCoeffs (metalFoamBackend.C:522-565) */
void orc_backend_set_coeffs(orc_backend* b, const double* diag,
                            const double* upper, const double* lower);
/* metalFoamBackend::pcg (metalFoamBackend.C:568-732) */
orc_stats orc_backend_pcg(orc_backend* b, const double* r, double target,
                          int32_t maxIter, int32_t iterationsPerSync,
                          int32_t chebOrder, double chebBeta,
                          double chebRatio);
/* metalFoamBackend::bicgstab (metalFoamBackend.C:735-959) */
orc_stats orc_backend_bicgstab(orc_backend* b, const double* r, double target,
                               int32_t maxIter);
const float* orc_backend_delta(const orc_backend* b);
/* Chebyshev constants of encCheb (metalFoamBackend.C:342-385):
 * c[0] = c1, then (c2, c3) per step i = 1..order-1 at c[2i-1], c[2i]. */
void orc_cheb_constants(int32_t order, double beta, double ratio, float* c);

/* Options of the driver's "metal" sub-dictionary plus the base controls. */
typedef struct
{
    double tolerance;
    double relTol;
    int32_t maxIter;
    int32_t minIter;
    int32_t maxRestarts;
    int32_t iterationsPerSync;
    int32_t deflate;          /* 0 auto, 1 on, 2 off */
    int32_t chebyshevOrder;
    double chebyshevRatio;
} orc_controls;

typedef struct
{
    double initialResidual;
    double finalResidual;
    int32_t nIterations;
    int32_t nRestarts;        /* value of `outer` after the restart loop */
    int32_t singular;
    int32_t converged;
    int32_t deflated;         /* deflation chosen at entry */
    int32_t polished;         /* hybrid polish switched to the exact diag */
    int32_t solved;           /* 0 when the entry test already converged */
    double chebBeta;
    double normFactor;
} orc_perf;

/* metalFoamSolver::solveImpl (metalFoamSolver.C:77-437) on the emulated
 * backend.  psi is updated in place.  lower == NULL: symmetric. */
int orc_metal_solve(int32_t n, int32_t nf, const int32_t* low,
                    const int32_t* upp, const int32_t* ownStart,
                    const int32_t* losort, const int32_t* losortStart,
                    const double* diag, const double* upper,
                    const double* lower, double* psi, const double* source,
                    int32_t useBiCGStab, const orc_controls* ctl,
                    orc_perf* perf);

/* ---------------------------------------------------------------- group 3 */

enum { ORC_PRECOND_NONE = 0, ORC_PRECOND_DIAGONAL = 1, ORC_PRECOND_DIC = 2 };

typedef struct
{
    double initialResidual;
    double finalResidual;
    int32_t nIterations;
    int32_t converged;
    int32_t singular;
} orc_foam_perf;

/* OpenFOAM's FP64 PCG (symmetric) -- the CPU path the plugin mirrors.
 * nthreads > 1 parallelises Amul and the vector reductions with OpenMP
 * (the DIC sweeps stay sequential). */
int orc_foam_pcg(int32_t n, int32_t nf, const int32_t* low,
                 const int32_t* upp, const int32_t* ownStart,
                 const int32_t* losort, const int32_t* losortStart,
                 const double* diag, const double* upper, double* psi,
                 const double* source, int32_t precond, double tolerance,
                 double relTol, int32_t maxIter, int32_t minIter,
                 int32_t nthreads, orc_foam_perf* perf);

/* OpenFOAM's FP64 PBiCGStab with the diagonal preconditioner. */
int orc_foam_pbicgstab(int32_t n, int32_t nf, const int32_t* low,
                       const int32_t* upp, const int32_t* ownStart,
                       const int32_t* losort, const int32_t* losortStart,
                       const double* diag, const double* upper,
                       const double* lower, double* psi,
                       const double* source, double tolerance, double relTol,
                       int32_t maxIter, int32_t minIter, int32_t nthreads,
                       orc_foam_perf* perf);

/* FP64 Jacobi-preconditioned CG (symmetric) or BiCGStab (lower != NULL)
 * run until ||b - A x||_2 <= tol_l2 * ||b||_2 (the accuracy oracle).
 * Returns iterations (negative if maxIter was reached). */
int orc_cg64(int32_t n, int32_t nf, const int32_t* low, const int32_t* upp,
             const int32_t* ownStart, const int32_t* losort,
             const int32_t* losortStart, const double* diag,
             const double* upper, const double* lower, double* x,
             const double* b, double tol_l2, int32_t maxIter,
             int32_t transpose, int32_t nthreads);

/* Face-parallel adjoint gradients of L(x) with x = A^{-1} b, given the
 * adjoint solution lambda = A^{-T} dL/dx:
 *   dL/dupper[f] = -lambda[l(f)] x[u(f)], dL/dlower[f] = -lambda[u(f)] x[l(f)],
 *   dL/ddiag[i]  = -lambda[i] x[i]. */
void orc_face_gradients(int32_t n, int32_t nf, const int32_t* low,
                        const int32_t* upp, const double* lambda,
                        const double* x, double* dUpper, double* dLower,
                        double* dDiag);

/* Row-parallel y = A x with OpenMP (order per row as orc_amul). */
void orc_amul_rows(int32_t n, const int32_t* low, const int32_t* upp,
                   const int32_t* ownStart, const int32_t* losort,
                   const int32_t* losortStart, const double* diag,
                   const double* upper, const double* lower, const double* x,
                   double* y, int32_t transpose, int32_t nthreads);

#ifdef __cplusplus
}
#endif

#endif
