/*
 * cudafoam.h -- C ABI of the B200 (sm_100a) Krylov hot path behind the
 * cudaPCG / cudaPBiCGStab lduMatrix::solver plugins.
 *
 * The library is a drop-in for the device backend and the FP64 driver of
 * the metal4Foam plugin (scotCW/metal4Foam).  Each entry point names the
 * reference interface it replaces:
 *
 *   backend   src/metal4Foam/backend/metalFoamBackend.H:37-115
 *   driver    src/metal4Foam/solvers/metalFoamSolver.H:60-108 (solveImpl)
 *   plugins   src/metal4Foam/solvers/metalPCG.H:47-92,
 *             src/metal4Foam/solvers/metalPBiCGStab.C:16-59
 *
 * Conventions
 *  - Plain pointers and sizes only.  Host pointers unless the name ends in
 *    _device (then CUDA device pointers on the context's device).
 *  - Every call returns an int status (CF_OK = 0).  No exception crosses the
 *    ABI; cf_last_error() returns a message for the calling thread.
 *  - Breakdown and stagnation are not errors: like the reference
 *    (metalFoamBackend::Stats, metalFoamBackend.H:41-50) they are reported as
 *    flags in the statistics structs.
 *  - One context per (mesh, field), the reference's cache key
 *    (metalFoamSolver.C:57-74).  A context is not shared between threads.
 *  - The caller owns host arrays; the context owns its device buffers.
 *  - Labels are int32 and scalars FP64 (the reference's static_asserts,
 *    metalFoamSolver.C:18-27).
 */
#ifndef CUDAFOAM_H
#define CUDAFOAM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CF_ABI_VERSION 1

/* status codes */
enum
{
    CF_OK = 0,
    CF_ERR_INVALID_ARG = 1,     /* null pointer, negative size, bad option */
    CF_ERR_BAD_ADDRESSING = 2,  /* faces not in LDU order / inconsistent   */
    CF_ERR_NO_TOPOLOGY = 3,     /* cf_set_topology not called              */
    CF_ERR_NO_COEFFS = 4,       /* cf_set_coeffs not called                */
    CF_ERR_CUDA = 5,            /* a CUDA runtime call failed              */
    CF_ERR_NO_DEVICE = 6,       /* no usable sm_100 device                 */
    CF_ERR_DEVICE_TIMEOUT = 7,  /* a bounded device-side wait expired      */
    CF_ERR_UNSUPPORTED = 8,     /* option combination not supported        */
    CF_ERR_TOO_LARGE = 9        /* size beyond a stated maximum            */
};

/* solver selection (the plugin names cudaPCG / cudaPBiCGStab) */
enum { CF_SOLVER_PCG = 0, CF_SOLVER_PBICGSTAB = 1 };

/* deflate on|off|auto (metalFoamSolver.C:170-190) */
enum { CF_DEFLATE_AUTO = 0, CF_DEFLATE_ON = 1, CF_DEFLATE_OFF = 2 };

/* preconditioner of the inner FP32 PCG: the reference's Chebyshev-Jacobi
 * polynomial of chebyshevOrder (default), or one aggregation multigrid
 * V-cycle (no counterpart in the reference, whose README.md:221-227 lists
 * GAMG as a limitation) */
enum { CF_PRECOND_CHEBYSHEV = 0, CF_PRECOND_GAMG = 1 };

/* internal cell ordering chosen at cf_set_topology */
enum { CF_REORDER_NONE = 0, CF_REORDER_RCM = 1, CF_REORDER_AUTO = 2 };

typedef struct cf_context cf_context;

/* metalFoamBackend::Stats (metalFoamBackend.H:41-50) */
typedef struct
{
    int32_t nIterations;      /* inner FP32 iterations performed          */
    int32_t converged;        /* hit the requested L1 target              */
    int32_t singular;         /* breakdown (non-finite scalars)           */
    int32_t stagnated;        /* 50 iterations without progress           */
    double finalResSum;       /* inner L1 sum |r| at exit (unnormalised)  */
    double tGpuSeconds;       /* device time of the inner loop            */
    double tWallSeconds;      /* host wall time of the call               */
} cf_inner_stats;

/* fvSolution controls: tolerance, relTol, maxIter, minIter (read by
 * OpenFOAM's lduMatrix::solver) and the plugin sub-dictionary keys
 * (metalFoamSolver.C:170-171,224-227,259-263). */
typedef struct
{
    double tolerance;          /* default 1e-6                             */
    double relTol;             /* default 0                                */
    int32_t maxIter;           /* default 1000                             */
    int32_t minIter;           /* default 0                                */
    int32_t maxRestarts;       /* default 8                                */
    int32_t iterationsPerSync; /* default 1: convergence test granularity  */
    int32_t deflate;           /* CF_DEFLATE_*, default AUTO (PCG only)    */
    int32_t chebyshevOrder;    /* default 8 (PCG); BiCGStab always 1       */
    double chebyshevRatio;     /* default 30                               */
    int32_t profile;           /* print a timing line per solve           */
    int32_t verbose;           /* print a residual line per restart        */
    int32_t graph;             /* 1 (default): inner loop as a device-side
                                  CUDA-graph while loop, no host sync per
                                  iteration; 0: one host sync per batch of
                                  iterationsPerSync, as the reference      */
    int32_t stagnationLimit;   /* inner iterations without a new minimum of
                                  sum|r| before the inner solve stops; 0
                                  (default) = 50, metalFoamBackend.C:606   */
    int32_t persistentMaxCells;/* with graph = 1 and > 0: meshes up to this
                                  many cells run each inner solve as ONE
                                  cooperative kernel (grid barriers between
                                  the phases of an iteration, bit-identical
                                  results; slower than the graph loop on
                                  B200, kept for comparison); for a batch
                                  (cf_batch_solve) whose rows all together
                                  are at most this many, the inner loop of
                                  every system runs as one cooperative
                                  launch per restart; 0 (default): never   */
    int32_t clusterMaxCells;   /* cudaPCG with graph = 1: meshes up to this
                                  many cells (at most 16384, one row per
                                  thread) whose columns lie mostly in their
                                  own CTA run each inner solve inside one
                                  thread-block cluster of up to 16 CTAs,
                                  the work vectors in distributed shared
                                  memory; 0 (default) = 16384, < 0 = never */
    int32_t preconditioner;    /* cudaPCG: CF_PRECOND_CHEBYSHEV (default) or
                                  CF_PRECOND_GAMG: z = M r is one symmetric
                                  V-cycle over aggregation levels (Galerkin
                                  coarse operators summed on the device each
                                  solve, Chebyshev-Jacobi smoothing on
                                  [beta/smootherRatio, beta], the coarsest
                                  level inverted densely); the FP64 driver
                                  is unchanged.  The V-cycle runs its own
                                  SELL-32 kernels whatever the SpMV launch
                                  shape (cf_set_spmv_config) is.           */
    int32_t nSweeps;           /* GAMG: Chebyshev degree of the smoother,
                                  2..8, default 3                          */
    int32_t nCellsInCoarsestLevel; /* GAMG: coarsening stops at this many
                                  cells or fewer, 1..128, default 128      */
    double scaleCorrection;    /* GAMG: fixed factor on every coarse-grid
                                  correction, in (0, 2) (the cycle stays
                                  symmetric positive definite), default
                                  1.8 (plain aggregation under-corrects)   */
    double smootherRatio;      /* GAMG: the smoother's Chebyshev interval is
                                  [beta/smootherRatio, beta] (> 1, default
                                  8); chebyshevRatio keeps its meaning for
                                  the Chebyshev-Jacobi preconditioner     */
} cf_options;

/* solverPerformance plus the reference's profile/verbose figures
 * (metalFoamSolver.C:127-128,363-365,417-426). */
typedef struct
{
    double initialResidual;    /* FP64 sum|b - A psi0| / normFactor        */
    double finalResidual;      /* FP64 sum|b - A psi|  / normFactor        */
    int32_t nIterations;       /* total inner iterations                   */
    int32_t nRestarts;         /* outer refinement passes - 1 (`outer`)    */
    int32_t converged;
    int32_t singular;
    int32_t stagnated;         /* last inner solve stagnated               */
    int32_t deflated;          /* constant-mode deflation chosen           */
    int32_t polished;          /* hybrid polish switched to the exact diag */
    int32_t solved;            /* 0: the entry test had already converged  */
    double normFactor;
    double chebBeta;           /* Gershgorin bound of D^-1 A               */
    double finalResSum32;      /* last inner L1 sum (unnormalised)         */
    double residualL2;         /* ||b - A psi||_2 / ||b||_2 at exit        */
    double tConvert;           /* seconds: coefficient staging             */
    double tInner;             /* seconds: host wall time of inner solves  */
    double tGpu;               /* seconds: device time of inner solves     */
    double tSolve;             /* seconds: device time of the whole solve  */
} cf_performance;

/* ------------------------------------------------------------ library */

int cf_abi_version(void);
/* message of the last failed call on this thread ("" if none) */
const char* cf_last_error(void);
/* fills defaults: tolerance 1e-6, relTol 0, maxIter 1000, minIter 0,
 * maxRestarts 8, iterationsPerSync 1, deflate auto, chebyshevOrder 8,
 * chebyshevRatio 30, graph 1, preconditioner Chebyshev, nSweeps 3,
 * nCellsInCoarsestLevel 128, scaleCorrection 1.8, smootherRatio 8 */
void cf_options_default(cf_options* opts);

/* ------------------------------------------------------------ context */

/* metalFoamBackend::metalFoamBackend / Impl::init (metalFoamBackend.C:192-282,
 * 422-430): binds a CUDA device (must be sm_100), creates a stream. */
int cf_context_create(cf_context** out, int32_t device);
int cf_context_destroy(cf_context* ctx);
/* metalFoamBackend::good (metalFoamBackend.H:106) */
int cf_context_good(const cf_context* ctx);
/* metalFoamBackend::description (metalFoamBackend.H:109) */
const char* cf_context_description(const cf_context* ctx);
/* Use the caller's cudaStream_t (e.g. torch.cuda.current_stream()) for
 * all later work of this context; NULL restores the context's own stream. */
int cf_context_set_stream(cf_context* ctx, void* stream);
/* Internal row ordering for the next cf_set_topology (default AUTO: RCM
 * for meshes above 65536 cells).  Results are returned in the caller's
 * ordering either way. */
int cf_context_set_reorder(cf_context* ctx, int32_t mode);
/* Polls a bounded device-side wait of this context (the grid barriers of
 * persistent inner solves, persistentMaxCells) makes before it gives up;
 * a wait that gives up ends the kernel and the solve returns
 * CF_ERR_DEVICE_TIMEOUT, leaving the context usable.  0 restores the
 * default, 2^24 polls of about 64 ns each.  No reference counterpart. */
int cf_context_set_wait_limit(cf_context* ctx, int64_t polls);
/* Number of kernels this context has launched so far (graph bodies are
 * counted once per executed iteration).  Diagnostic; no reference
 * counterpart. */
int cf_context_kernel_launches(const cf_context* ctx, long long* count);

/* ------------------------------------------------------------ matrix */

/* metalFoamBackend::setTopology (metalFoamBackend.H:60-69,
 * metalFoamBackend.C:454-519).  The five lduAddressing arrays; validated
 * (ranges, LDU order, consistency of ownerStart/losort/losortStart) and
 * cached on (nCells, nFaces, lowAddr, uppAddr) identity like the
 * reference.  Builds the device layout once per mesh. */
int cf_set_topology(cf_context* ctx, int32_t nCells, int32_t nFaces,
                    const int32_t* lowAddr, const int32_t* uppAddr,
                    const int32_t* ownStartAddr, const int32_t* losortAddr,
                    const int32_t* losortStartAddr);

/* metalFoamBackend::setCoeffs (metalFoamBackend.H:74-79,
 * metalFoamBackend.C:522-565).  FP64 diag[nCells], upper[nFaces],
 * lower[nFaces] (NULL: symmetric).  Keeps FP64 copies on the device and
 * stages FP32 copies plus rD = float(1/diag) there.  *tConvert (may be
 * NULL) receives the seconds spent, like the reference's return value. */
int cf_set_coeffs(cf_context* ctx, const double* diag, const double* upper,
                  const double* lower, double* tConvert);
/* Same from device pointers (no host copy). */
int cf_set_coeffs_device(cf_context* ctx, const double* diag,
                         const double* upper, const double* lower);

/* ------------------------------------------------------------ inner solves */

/* metalFoamBackend::pcg (metalFoamBackend.H:83-92, .C:568-732): FP32 PCG on
 * A delta = r with Jacobi (chebOrder 1) or Chebyshev-Jacobi (chebOrder > 1)
 * preconditioning on the FP32 coefficients staged last, stopping on
 * sum|r| <= targetResSum, breakdown, 50 iterations without progress or
 * maxIter; the minimum-residual iterate is kept.  r is FP64 (host). */
int cf_pcg(cf_context* ctx, const double* r, double targetResSum,
           int32_t maxIter, int32_t iterationsPerSync, int32_t chebOrder,
           double chebBeta, double chebRatio, cf_inner_stats* stats);
/* metalFoamBackend::bicgstab (metalFoamBackend.H:95-100, .C:735-959) */
int cf_bicgstab(cf_context* ctx, const double* r, double targetResSum,
                int32_t maxIter, cf_inner_stats* stats);
/* metalFoamBackend::delta (metalFoamBackend.H:103): copies the FP32
 * correction of the last inner solve (caller's cell order). */
int cf_delta(cf_context* ctx, float* delta);

/* ------------------------------------------------------------ full solve */

/* metalFoamSolver::solveImpl (metalFoamSolver.H:78-85, .C:77-437) with
 * every FP64 step on the device: residual r = b - A psi, normFactor, the
 * L1 convergence tests, row sums u = A 1, deflation decision and deflated
 * diagonal, Gershgorin bound, zero-mean inner right-hand side, psi += delta,
 * constant-mode shift, hybrid polish.  psi is updated in place.  Uses the
 * coefficients of the last cf_set_coeffs. */
int cf_solve(cf_context* ctx, int32_t solver, double* psi,
             const double* source, const cf_options* opts,
             cf_performance* perf);
/* Same with device pointers (psi, source on the context's device). */
int cf_solve_device(cf_context* ctx, int32_t solver, double* psi,
                    const double* source, const cf_options* opts,
                    cf_performance* perf);
/* FP64 residual field b - A psi of the last cf_solve (which = 0: at entry,
 * 1: at exit), caller's cell order, for lduMatrix::setResidualField
 * (metalFoamSolver.C:112-117,429-434). */
int cf_residual(cf_context* ctx, int32_t which, double* r);

/* ------------------------------------------------------------ adjoint */
/* No counterpart in the reference (the design's differentiation row).
 * For x = A^{-1} b and a loss L(x): lambda = A^{-T} dL/dx and
 *   dL/db = lambda, dL/ddiag[i] = -lambda[i] x[i],
 *   dL/dupper[f] = -lambda[l(f)] x[u(f)], dL/dlower[f] = -lambda[u(f)] x[l(f)]
 * (upper[f] = A[l(f),u(f)], lower[f] = A[u(f),l(f)]).  A^T in LDU form is A
 * with upper and lower exchanged: the transpose solve reuses the forward
 * kernels on restaged values. */

/* on != 0: stage A^T for the following solves/operators; 0: back to A. */
int cf_set_transpose(cf_context* ctx, int32_t on);
/* The gradient pass alone (face order / caller's cell order). */
int cf_face_gradients(cf_context* ctx, const double* lambda, const double* x,
                      double* dUpper, double* dLower, double* dDiag);
int cf_face_gradients_device(cf_context* ctx, const double* lambda,
                             const double* x, double* dUpper, double* dLower,
                             double* dDiag);
/* Adjoint solve (A^T lambda = dLdx from lambda0 = 0, same driver and
 * options as cf_solve) followed by the gradient pass; leaves A staged. */
int cf_solve_adjoint(cf_context* ctx, int32_t solver, const double* x,
                     const double* dLdx, double* lambda, double* dUpper,
                     double* dLower, double* dDiag, const cf_options* opts,
                     cf_performance* perf);
int cf_solve_adjoint_device(cf_context* ctx, int32_t solver, const double* x,
                            const double* dLdx, double* lambda,
                            double* dUpper, double* dLower, double* dDiag,
                            const cf_options* opts, cf_performance* perf);

/* ------------------------------------------------------------ batches */
/* No counterpart in the reference (the design's batching row).  A batch
 * holds many independent symmetric pressure systems of any sizes and
 * solves them together with cudaPCG semantics per system (same driver
 * decisions, same stopping tests as cf_solve on each system alone): every
 * phase of the iteration is one launch over all still-active systems and
 * the iterations run in a device-side CUDA-graph loop until the last
 * system has finished. */
typedef struct cf_batch cf_batch;

int cf_batch_create(cf_batch** out, int32_t device);
int cf_batch_destroy(cf_batch* batch);
int cf_batch_set_stream(cf_batch* batch, void* stream);
int cf_batch_kernel_launches(const cf_batch* batch, long long* count);
/* Adds one system (its lduAddressing, copied and validated); *index is its
 * position.  All systems are added before cf_batch_finalize. */
int cf_batch_add_system(cf_batch* batch, int32_t nCells, int32_t nFaces,
                        const int32_t* lowAddr, const int32_t* uppAddr,
                        const int32_t* ownStartAddr, const int32_t* losortAddr,
                        const int32_t* losortStartAddr, int32_t* index);
/* Systems of at least minCells cells (0, the default: three 256-row blocks
 * per SM, numSMs x 768, 113,664 on B200; < 0: never) are solved as single
 * solves (a context of their own, cf_solve's path and result) on their own
 * host thread and stream, concurrently with the batched launches of the
 * rest: a system that keeps several blocks busy on every SM gains little
 * from sharing a launch, while the small ones gain from it.  Call before
 * cf_batch_finalize. */
int cf_batch_set_solo_cells(cf_batch* batch, int32_t minCells);
/* Lays all systems out on the device (reorder: CF_REORDER_*, per system). */
int cf_batch_finalize(cf_batch* batch, int32_t reorder);
/* FP64 coefficients of system `index` (lower must be NULL: symmetric). */
int cf_batch_set_coeffs(cf_batch* batch, int32_t index, const double* diag,
                        const double* upper, const double* lower);
int cf_batch_set_coeffs_device(cf_batch* batch, int32_t index,
                               const double* diag, const double* upper,
                               const double* lower);
/* Solves every system: psi[i] (in/out) and source[i] per system (host
 * pointers; _device: device pointers), perf[i] per system.  solver must be
 * CF_SOLVER_PCG. */
int cf_batch_solve(cf_batch* batch, int32_t solver, double* const* psi,
                   const double* const* source, const cf_options* opts,
                   cf_performance* perf);
int cf_batch_solve_device(cf_batch* batch, int32_t solver, double* const* psi,
                          const double* const* source, const cf_options* opts,
                          cf_performance* perf);

/* ------------------------------------------------------------ several RHS */
/* No counterpart in the reference (the design's multi-RHS row): the
 * reference solves the components of a vector equation one after another
 * (fvMatrix<vector>::solveSegregated calls the scalar solver per
 * component).  cf_solve_multi solves nrhs systems A psi_k = source_k on the
 * matrix of the last cf_set_coeffs together: psi and source hold nrhs
 * component fields of nCells each (component k at offset k*nCells), perf
 * has nrhs entries.  Two forms, chosen by the context's rhsTile
 * (cf_set_spmv_config):
 *   rhsTile 0 (default): the components run at once as single solves, up
 *     to 8 side by side, each on its own stream and host thread, with the
 *     matrix stored once (the context's arrays, read by all).  The first
 *     call allocates the vectors of min(nrhs, 8) solves (116 bytes per
 *     cell each), kept until the topology changes or the context is
 *     destroyed;
 *   rhsTile 1..4: fused passes in which every SpMV reads the matrix once
 *     for up to rhsTile components.
 * In both, each component keeps its own scalars, early exit, stopping tests
 * and restarts, and its results equal those of cf_solve on that component
 * alone, bit for bit.  solver must be CF_SOLVER_PBICGSTAB (momentum).
 * cf_residual keeps referring to the last single solve. */
int cf_solve_multi(cf_context* ctx, int32_t solver, int32_t nrhs, double* psi,
                   const double* source, const cf_options* opts,
                   cf_performance* perf);
int cf_solve_multi_device(cf_context* ctx, int32_t solver, int32_t nrhs,
                          double* psi, const double* source,
                          const cf_options* opts, cf_performance* perf);

/* ------------------------------------------------------------ operators */

/* y = A x in FP64 with lduMatrix::Amul's per-row summation order
 * (metalFoamSolver.C:109,333); transpose != 0 applies A^T (upper and lower
 * exchanged).  Host pointers, caller's cell order. */
int cf_amul(cf_context* ctx, const double* x, double* y, int32_t transpose);
/* y = A x in FP32 on the staged FP32 coefficients, with the summation
 * order of the reference's ldu_spmv_dotw kernel
 * (metalFoamKernels.metal:64-109), and dot = sum w.y (FP64 accumulation).
 * w may be NULL (dot then not computed). */
int cf_spmv32(cf_context* ctx, const float* x, const float* w, float* y,
              double* dot);
/* z = Chebyshev-Jacobi apply of the given order to r on the spectrum
 * [beta/ratio, beta] (encCheb, metalFoamBackend.C:342-385), FP32. */
int cf_cheb_apply(cf_context* ctx, const float* r, float* z, int32_t order,
                  double beta, double ratio);

/* ------------------------------------------------------------ measurement */

enum
{
    CF_KERNEL_CHEB_STEP = 0,   /* fused SpMV + Chebyshev step (cudaPCG bulk) */
    CF_KERNEL_SPMV32 = 1,      /* FP32 SpMV with fused dot                   */
    CF_KERNEL_PCG_P_SPMV = 2,  /* p-update fused into the SpMV + p.Ap        */
    CF_KERNEL_PCG_UPDATE = 3,  /* delta/residual update + L1 + next apply    */
    CF_KERNEL_AMUL64 = 4,      /* FP64 refinement residual SpMV              */
    CF_KERNEL_CHEB_STEP_INNER = 5, /* the Chebyshev steps inside `reps` full
                                     PCG iterations (order 8), each step
                                     bracketed by events: the cache state of
                                     a real solve, not of one kernel repeated;
                                     starts from the last solve's inner
                                     right-hand side (CF_ERR_INVALID_ARG when
                                     that is zero, e.g. before any solve)   */
    CF_KERNEL_SPMV32_COLD = 6  /* FP32 SpMV + dot with L2 flushed (256 MB
                                  read) before every timed launch           */
};
/* Launches one hot kernel `reps` times back to back on the context's stream
 * over the operands of the last solve (work vectors are overwritten, the
 * returned solution is not) and returns the average device time per launch
 * from CUDA events recorded on that stream.  Diagnostic; no reference
 * counterpart. */
int cf_time_kernel(cf_context* ctx, int32_t which, int32_t reps,
                   double* msPerLaunch);

/* ------------------------------------------------------------ kernel check */
/* One launch of a fused inner-iteration kernel on caller-supplied vectors
 * and scalars, exactly as the inner loop launches it (same kernel, launch
 * shape and buffers; iteration 0 of a live solve), for comparison with the
 * reference's unfused kernel sequence (metalFoamKernels.metal:64-276,
 * 372-458).  Diagnostic; no reference counterpart.  Host pointers, nCells
 * floats each, caller's cell order; the FP32 matrix, diag and rD are those
 * staged by the last cf_set_coeffs / solve.  alpha, beta, omega are the
 * solver scalars (the kernel rounds them to FP32 as the loop does).  sums
 * receives the step's reductions (products of FP32 values accumulated in
 * FP64).  The context's work vectors are overwritten.
 *
 *   CF_STEP_CHEB        in zIn, wIn, rA; chebOrder, chebStep (1..order-1),
 *                       chebBeta, chebRatio -> v = A zIn,
 *                       wOut = c2 wIn + c3 rD (rA - v), zOut = zIn + wOut;
 *                       sums[0] = zOut.rA on the last step
 *   CF_STEP_PCG_P_SPMV  in wA, pOld; beta -> p = wA + beta pOld, q = A p;
 *                       sums[0] = p.q
 *   CF_STEP_PCG_UPDATE  in delta, p, rA, q; alpha; chebOrder (1: Jacobi)
 *                       -> deltaNext = delta + alpha p, rAOut = rA - alpha q,
 *                       wAOut = c1 rD rAOut (Chebyshev start) or
 *                       rAOut rD (Jacobi); sums[0] = sum|rAOut|,
 *                       sums[1] = wAOut.rAOut (Jacobi)
 *   CF_STEP_BICG_AB     in rA, pOld, AyAOld, rA0; beta, omega
 *                       -> p = rA + beta (pOld - omega AyAOld), yA = rD p,
 *                       AyA = A yA; sums[0] = rA0.AyA
 *   CF_STEP_BICG_CD     in rA, AyA; alpha -> sA = rA - alpha AyA,
 *                       zA = rD sA, tA = A zA; sums = sum|sA|, sA.tA, tA.tA
 *   CF_STEP_BICG_E      in delta, yA, zA, sA, tA, rA0; alpha, omega
 *                       -> deltaNext = delta + (alpha yA + omega zA),
 *                       rAOut = sA - omega tA; sums = sum|rAOut|, rA0.rAOut
 */
enum
{
    CF_STEP_CHEB = 0,
    CF_STEP_PCG_P_SPMV = 1,
    CF_STEP_PCG_UPDATE = 2,
    CF_STEP_BICG_AB = 3,
    CF_STEP_BICG_CD = 4,
    CF_STEP_BICG_E = 5
};

typedef struct cf_step_io
{
    const float* rA;
    const float* rA0;
    const float* wA;
    const float* pOld;
    const float* AyAOld;
    const float* delta;
    const float* zIn;
    const float* wIn;
    float* p;             /* in for PCG_UPDATE, out for P_SPMV and BICG_AB   */
    float* q;             /* in for PCG_UPDATE, out for P_SPMV               */
    float* yA;            /* in for BICG_E, out for BICG_AB                  */
    float* AyA;           /* in for BICG_CD, out for BICG_AB                 */
    float* sA;            /* in for BICG_E, out for BICG_CD                  */
    float* zA;            /* in for BICG_E, out for BICG_CD                  */
    float* tA;            /* in for BICG_E, out for BICG_CD                  */
    float* deltaNext;
    float* rAOut;
    float* wAOut;
    float* wOut;
    float* zOut;
    double alpha, beta, omega;
    int32_t chebOrder;
    int32_t chebStep;
    double chebBeta;
    double chebRatio;
    double sums[3];
} cf_step_io;

int cf_inner_step(cf_context* ctx, int32_t step, cf_step_io* io);

/* ------------------------------------------------------------ autotuning */
/* No counterpart in the reference (the design's autotuner row).  The SpMV
 * inside the FP32 Krylov kernels (Chebyshev steps, p-update SpMV, both
 * BiCGStab SpMVs, cf_spmv32, cf_cheb_apply) runs in one of several launch
 * shapes:
 *   layout CF_LAYOUT_SELL32: the SELL-32 copy of the matrix, one row per
 *     thread (rowsPerWarp 32);
 *   layout CF_LAYOUT_LDU: the reference's own addressing read directly
 *     (ownerStartAddr ranges of upperAddr / upper, then losortStartAddr
 *     ranges of losortAddr -> lowerAddr / lower, metalFoamKernels.metal:64-109),
 *     rowsPerWarp 32 (row per thread), 8, 4 or 1 (warp per row: the lanes
 *     of a row load its entries and form the products together);
 *   blockSize 128, 256 or 512 threads; rhsTile 1..4 components per fused
 *   pass of cf_solve_multi, or 0 for its concurrent form (components as
 *   single solves side by side).
 * Every shape forms each row of A x with the same operations in the same
 * order (the products of a row are added one by one in the reference's
 * entry order), so A x is bit-identical across shapes; dot products fold
 * their partial sums in a shape-dependent order.  The default is SELL32,
 * 32 rows per warp, 256 threads, rhsTile 0, indexBits 16.  cf_autotune times
 * the layouts and, when rhsTile is 1..4, the fused tile; it keeps rhsTile 0.
 * The batched kernels (cf_batch_*) and the fused multi-RHS kernels always use
 * the default layout; the concurrent multi-RHS form uses the context's. */
enum
{
    CF_LAYOUT_SELL32 = 0,
    CF_LAYOUT_LDU = 1
};

typedef struct cf_spmv_config
{
    int32_t layout;
    int32_t rowsPerWarp;
    int32_t blockSize;
    int32_t rhsTile;
    int32_t indexBits;      /* SELL32 column stream: 16 (row-relative offsets,
                               used when every column of the reordered matrix
                               lies within 32767 rows of its row; otherwise
                               the 32-bit stream) or 32; ignored for LDU     */
} cf_spmv_config;

typedef struct cf_tune_entry
{
    cf_spmv_config config;
    double msPerLaunch;     /* FP32 SpMV + dot, CUDA events, inputs in HBM  */
} cf_tune_entry;

int cf_spmv_config_default(cf_spmv_config* cfg);
int cf_get_spmv_config(cf_context* ctx, cf_spmv_config* cfg);
/* Validates and applies; CF_ERR_UNSUPPORTED for a shape not in the list. */
int cf_set_spmv_config(cf_context* ctx, const cf_spmv_config* cfg);
/* Times the FP32 SpMV in every shape on the context's matrix (reps launches
 * each after one warm-up) and the multi-RHS SpMV for 1..4 components, then
 * writes the fastest shape (and the RHS tile with the least time per
 * component) to *best; apply != 0 also makes it the context's shape.
 * table (capacity entries, may be NULL) receives every timing; *count the
 * number of shapes timed. */
int cf_autotune(cf_context* ctx, int32_t reps, int32_t apply, cf_spmv_config* best,
                cf_tune_entry* table, int32_t capacity, int32_t* count);

/* ------------------------------------------------------------ many systems */
/* Independent systems, one context each (topology set), solved concurrently:
 * `streams` host threads (1..64), each with its own CUDA stream, take the
 * systems largest first and, for each, stage the coefficients when diag is
 * not NULL (cf_set_coeffs_device with diag[i], upper[i], lower ? lower[i] :
 * NULL) and run cf_solve_device(ctx[i], solver, psi[i], source[i], opts,
 * &perf[i]).  All contexts must be on one device (CF_ERR_INVALID_ARG
 * otherwise); all pointers are device pointers on it; work queued earlier on
 * any stream of that device completes first, and everything is complete on
 * return.  Every
 * system gets exactly what cf_solve_device on it alone returns.  A context
 * may appear once.  No counterpart in the reference. */
int cf_solve_many_device(cf_context* const* ctx, int32_t count, int32_t solver,
                         double* const* psi, const double* const* source,
                         const double* const* diag, const double* const* upper,
                         const double* const* lower, const cf_options* opts, int32_t streams,
                         cf_performance* perf);

/* ------------------------------------------------------------ subdomains */
/* A subdomain of a decomposed mesh solved together with its neighbours
 * across processor interfaces.  The reference rejects coupled interfaces
 * (metalFoamSolver.C:89-99); these entry points have no counterpart there.
 * Each subdomain (one per MPI rank, GPU or thread) holds its own LDU matrix
 * in the lduAddressing form of cf_set_topology plus nInterfaces processor
 * interfaces in OpenFOAM's form: interface p faces subdomain neighbour[p];
 * faceCells (nFaces[0] + nFaces[1] + ... entries, interface after
 * interface) are this side's cells of the interface faces, listed in the
 * same face order as the neighbour lists them; interfaceCoeffs (same
 * layout) are the interfaceBouCoeffs: row faceCells[k] of A psi gets
 * -interfaceCoeffs[k] * psi_neighbour[k], after the internal faces, as
 * lduMatrix::Amul's updateMatrixInterfaces does.  At most one interface per
 * neighbouring subdomain.
 *
 * Communication is the caller's (MPI/Pstream, NCCL, or the in-process hub
 * of cf_comm_local_create).  With hostBuffers = 0 both callbacks receive
 * device pointers on the subdomain's device and the subdomain's
 * cudaStream_t; they may complete the work before returning or enqueue it
 * on that stream (NCCL), as long as work enqueued on the stream afterwards
 * sees the result.  With hostBuffers != 0 they receive host pointers
 * (pinned staging buffers the library fills before the call and reads back
 * after it) and must complete the work before returning -- the form for
 * MPI without CUDA awareness.  They return 0 on success.  Every subdomain
 * calls them in the same order with the same counts (all decisions depend
 * on globally reduced values). */
typedef struct cf_comm
{
    void* user;
    /* in place over all subdomains: op 0 sum, 1 max, of `count` doubles */
    int (*allreduce)(void* user, double* values, int32_t count, int32_t op, void* stream);
    /* for every interface p: send[p] (nFaces[p] elements of elemBytes,
     * this side's face order) to subdomain neighbour[p]; that subdomain's
     * values for the same faces into recv[p] */
    int (*exchange)(void* user, int32_t nInterfaces, const int32_t* neighbour,
                    const int32_t* nFaces, int32_t elemBytes, const void* const* send,
                    void* const* recv, void* stream);
    /* optional: called when this subdomain's solve fails, so the others
     * stop waiting for it */
    void (*abort)(void* user);
    /* != 0: the callbacks get host buffers (see above); 0: device buffers */
    int32_t hostBuffers;
} cf_comm;

typedef struct cf_subdomain cf_subdomain;

int cf_subdomain_create(cf_subdomain** out, int32_t device);
int cf_subdomain_destroy(cf_subdomain* sub);
int cf_subdomain_set_stream(cf_subdomain* sub, void* stream);
int cf_subdomain_kernel_launches(const cf_subdomain* sub, long long* count);
/* internal addressing (validated as by cf_set_topology) and interfaces;
 * reorder: CF_REORDER_* of the internal cells */
int cf_subdomain_set_topology(cf_subdomain* sub, int32_t nCells, int32_t nFaces,
                              const int32_t* lowAddr, const int32_t* uppAddr,
                              const int32_t* ownStartAddr, const int32_t* losortAddr,
                              const int32_t* losortStartAddr, int32_t nInterfaces,
                              const int32_t* neighbour, const int32_t* nInterfaceFaces,
                              const int32_t* faceCells, int32_t reorder);
/* FP64 diag, upper, lower (NULL: symmetric) and interfaceCoeffs (host) */
int cf_subdomain_set_coeffs(cf_subdomain* sub, const double* diag, const double* upper,
                            const double* lower, const double* interfaceCoeffs);
/* cf_solve's driver and inner solves over all subdomains (every sum global,
 * halos exchanged before each SpMV; preconditioner Chebyshev-Jacobi; one
 * host synchronisation per inner iteration); psi (in/out) and source are
 * this subdomain's host arrays.  With no interfaces and one subdomain the
 * result equals cf_solve's bit for bit. */
int cf_subdomain_solve(cf_subdomain* sub, int32_t solver, double* psi, const double* source,
                       const cf_options* opts, const cf_comm* comm, cf_performance* perf);

/* An in-process communicator for nRanks subdomains solved by nRanks host
 * threads of one process (one GPU or several): fills comms[0..nRanks-1].
 * The threads meet at host barriers; a thread that waits longer than
 * timeoutSeconds, or a failed solve (abort), makes every later call of
 * every rank fail instead of waiting. */
int cf_comm_local_create(int32_t nRanks, double timeoutSeconds, cf_comm* comms);
int cf_comm_local_destroy(int32_t nRanks, cf_comm* comms);

/* ------------------------------------------------------------ GAMG */
/* Cells of every level of the context's multigrid hierarchy (built by the
 * first cudaPCG solve with CF_PRECOND_GAMG on the current topology; level 0
 * is the mesh): *levels receives the number of levels (0 before any GAMG
 * solve), cells[0..min(levels, capacity)-1] their sizes. */
int cf_gamg_levels(cf_context* ctx, int32_t* cells, int32_t capacity, int32_t* levels);
/* Level `level` (>= 1) of that hierarchy as an LDU matrix, for inspection:
 * *nFaces its faces; agg[i] (cells of level - 1; for level 1 indexed by the
 * caller's cell numbering) the cell of `level` that cell i belongs to;
 * diag[cells(level)], upper[nFaces] the Galerkin operator P^T A P as the
 * last GAMG solve staged it (FP64); lowerAddr/upperAddr[nFaces] its faces
 * (owner < neighbour, sorted).  Any array may be NULL (only *nFaces then). */
int cf_gamg_export(cf_context* ctx, int32_t level, int32_t* nFaces, int32_t* agg, double* diag,
                   double* upper, int32_t* lowerAddr, int32_t* upperAddr);

/* ------------------------------------------------------------ no allocation */

/* y = A x and *dot = sum w.y for callers that cannot allocate device memory:
 * code running inside someone else's CUDA-graph capture, solver threads
 * that must not take the allocator's locks, or frameworks that hand out only
 * their own pre-allocated buffers.  No counterpart in the reference.
 *
 * Everything is a device pointer on the current device and is owned by the
 * caller: the LDU arrays as cf_set_topology takes them (none may be NULL;
 * a mesh without faces passes any valid device pointer for the face
 * arrays), FP32 coefficients (lower NULL: symmetric), x, w (NULL: dot = 0),
 * y and dot (one double; NULL: no dot).  NULL where a pointer is required
 * returns CF_ERR_INVALID_ARG before anything is launched.  The row sums use
 * the reference kernel's order (diagonal, owner-side faces, then losort
 * faces).  The call is asynchronous on `stream` (a cudaStream_t, NULL: the
 * default stream) and calls no cudaMalloc, cudaFree or allocating library
 * routine: the per-block partial sums live in a fixed file-scope device
 * array of 65,536 doubles plus one 256-byte line, which every GPU that loads
 * the library keeps until the process exits.  Hence nCells is limited to
 * 16,777,216; larger sizes return CF_ERR_TOO_LARGE before anything is
 * launched.  The first call in a CUDA context looks up that array's device
 * address (cudaGetSymbolAddress) and caches it for the context: make it
 * before any stream capture (made while `stream` is capturing, it returns
 * CF_ERR_UNSUPPORTED and launches nothing).  All calls on a device share the
 * array, so calls whose kernels overlap on the GPU (different streams
 * without ordering) race and give wrong dot products. */
int cf_ldu_spmv_dot_noalloc(int32_t nCells, const float* diag,
                            const float* upper, const float* lower,
                            const int32_t* lowAddr, const int32_t* uppAddr,
                            const int32_t* ownStartAddr,
                            const int32_t* losortAddr,
                            const int32_t* losortStartAddr, const float* x,
                            const float* w, float* y, double* dot,
                            void* stream);

#ifdef __cplusplus
}
#endif

#endif
