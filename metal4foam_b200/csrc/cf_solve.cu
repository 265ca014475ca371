// cf_solve.cu -- inner FP32 Krylov loops (device-driven), the FP64
// refinement driver, and the operator entry points of the C ABI.
#include "cudafoam.h"
#include "cf_host.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

using namespace cf;

#define CF_CUDA(call)                                                           \
    do                                                                          \
    {                                                                           \
        cudaError_t e_ = (call);                                                \
        if (e_ != cudaSuccess)                                                  \
            return fail(CF_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define CF_TRY(expr)                  \
    do                                \
    {                                 \
        int rc_ = (expr);             \
        if (rc_ != CF_OK) return rc_; \
    } while (0)

#define CF_LAUNCH()                                                             \
    do                                                                          \
    {                                                                           \
        cudaError_t e_ = cudaGetLastError();                                    \
        if (e_ != cudaSuccess)                                                  \
            return fail(CF_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e_)); \
        c->launches++;                                                          \
    } while (0)

namespace {

constexpr int MW = MAXW_UNROLL;

int chebz(int j) { return j & 1; }

// One PCG iteration (Chebyshev steps, p-update+SpMV, update); identical
// for graph capture and for host-synchronised execution.
int launch_pcg_body(cf_context* c, int order, cudaGraphConditionalHandle h, int useCond,
                    int* kernels)
{
    if (c->amgActive) return launch_amg_body(c, order, h, useCond, kernels);
    const DevSell A = sell_of(c);
    const PcgBufs B = pcg_bufs(c);
    cudaStream_t s = c->stream;
    const float* wA = B.W0;
    int nk = 0;
    if (order > 1)
    {
        float* Z[2] = {B.Z0, B.Z1};
        for (int j = 1; j < order; ++j)
        {
            const float* zin = (j == 1) ? B.W0 : Z[chebz(j - 1)];
            const float* win = (j == 1) ? B.W0 : B.W1;
            float* zout = Z[chebz(j)];
            if (!spmv_default(c))
            {
                CF_TRY(launch_cheb_step_v(c, j == order - 1, B, zin, win, B.W1, zout, j));
                ++nk;
                continue;
            }
            if (j == order - 1)
            {
                auto fn = cheb_step_kernel<true>(A);
                fn<<<grid_for(c, (const void*)fn, c->n), NT, 0, s>>>(A, B, zin, win, B.W1, zout, j,
                                                                    c->d_st, c->d_part);
            }
            else
            {
                auto fn = cheb_step_kernel<false>(A);
                fn<<<rows_grid(c->n), NT, 0, s>>>(A, B, zin, win, B.W1, zout, j, c->d_st,
                                                  c->d_part);
            }
            CF_LAUNCH();
            ++nk;
        }
        wA = Z[chebz(order - 1)];
    }
    if (!spmv_default(c))
    {
        CF_TRY(launch_pcg_p_spmv_v(c, B, wA));
        ++nk;
    }
    else
    {
        auto fn = pcg_p_spmv_kernel(A);
        fn<<<grid_for(c, (const void*)fn, c->n), NT, 0, s>>>(A, B, wA, c->d_st, c->d_part);
        CF_LAUNCH();
        ++nk;
    }
    if (order > 1)
    {
        auto fn = k_pcg_update<true>;
        fn<<<grid_for(c, (const void*)fn, c->n), NT, 0, s>>>(B, c->d_st, c->d_part, h, useCond);
    }
    else
    {
        auto fn = k_pcg_update<false>;
        fn<<<grid_for(c, (const void*)fn, c->n), NT, 0, s>>>(B, c->d_st, c->d_part, h, useCond);
    }
    CF_LAUNCH();
    ++nk;
    if (kernels) *kernels = nk;
    return CF_OK;
}

int launch_bicg_body(cf_context* c, cudaGraphConditionalHandle h, int useCond, int* kernels)
{
    const DevSell A = sell_of(c);
    const BicgBufs B = bicg_bufs(c);
    cudaStream_t s = c->stream;
    if (!spmv_default(c))
    {
        CF_TRY(launch_bicg_ab_v(c, B));
        CF_TRY(launch_bicg_cd_v(c, B, h, useCond));
    }
    else
    {
        auto fab = bicg_ab_kernel(A);
        fab<<<grid_for(c, (const void*)fab, c->n), NT, 0, s>>>(A, B, c->d_st, c->d_part);
        CF_LAUNCH();
        auto fcd = bicg_cd_kernel(A);
        fcd<<<grid_for(c, (const void*)fcd, c->n), NT, 0, s>>>(A, B, c->d_st, c->d_part, h,
                                                              useCond);
        CF_LAUNCH();
    }
    k_bicg_e<<<grid_for(c, (const void*)k_bicg_e, c->n), NT, 0, s>>>(B, c->d_st, c->d_part, h,
                                                                    useCond);
    CF_LAUNCH();
    if (kernels) *kernels = 3;
    return CF_OK;
}

// Instantiate (once per topology, kind and order) a graph holding one
// conditional WHILE node whose body is one iteration; the last kernel of
// the body sets the condition from the device-side convergence state.
int get_graph(cf_context* c, int kind, int order, cudaGraphExec_t* out, int* bodyKernels)
{
    // (kind 2: PCG whose preconditioner is the multigrid V-cycle)
    const auto key = std::make_pair(kind == 0 && c->amgActive ? 2 : kind, kind == 0 ? order : 1);
    auto it = c->graphs.find(key);
    if (it != c->graphs.end())
    {
        *out = it->second;
        *bodyKernels = c->graphKernels[key];
        return CF_OK;
    }
    cudaGraph_t g = nullptr;
    CF_CUDA(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle h;
    cudaError_t e = cudaGraphConditionalHandleCreate(&h, g, 1u, cudaGraphCondAssignDefault);
    if (e != cudaSuccess)
    {
        cudaGraphDestroy(g);
        return fail(CF_ERR_CUDA, std::string("cudaGraphConditionalHandleCreate: ") +
                                     cudaGetErrorString(e));
    }
    // the struct holds a union with constructors: zero-filled raw storage
    alignas(cudaGraphNodeParams) unsigned char cpStorage[sizeof(cudaGraphNodeParams)];
    std::memset(cpStorage, 0, sizeof(cpStorage));
    cudaGraphNodeParams& cp = *reinterpret_cast<cudaGraphNodeParams*>(cpStorage);
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    e = cudaGraphAddNode(&node, g, nullptr, 0, &cp);
    if (e != cudaSuccess)
    {
        cudaGraphDestroy(g);
        return fail(CF_ERR_CUDA, std::string("cudaGraphAddNode(conditional): ") +
                                     cudaGetErrorString(e));
    }
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    e = cudaStreamBeginCaptureToGraph(c->stream, body, nullptr, nullptr, 0,
                                      cudaStreamCaptureModeRelaxed);
    if (e != cudaSuccess)
    {
        cudaGraphDestroy(g);
        return fail(CF_ERR_CUDA, std::string("cudaStreamBeginCaptureToGraph: ") +
                                     cudaGetErrorString(e));
    }
    const long long before = c->launches;
    int nk = 0;
    int rc = kind == 0 ? launch_pcg_body(c, order, h, 1, &nk) : launch_bicg_body(c, h, 1, &nk);
    c->launches = before;
    cudaGraph_t captured = nullptr;
    e = cudaStreamEndCapture(c->stream, &captured);
    if (rc != CF_OK || e != cudaSuccess)
    {
        cudaGraphDestroy(g);
        if (rc != CF_OK) return rc;
        return fail(CF_ERR_CUDA, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e));
    }
    cudaGraphExec_t exec = nullptr;
    e = cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess)
        return fail(CF_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    c->graphs[key] = exec;
    c->graphKernels[key] = nk;
    *out = exec;
    *bodyKernels = nk;
    return CF_OK;
}

// The inner solve on the staged FP32 operator.  r64 (internal order) holds
// the right-hand side; `mean` (device, may be NULL) is subtracted from it.
// kind 0: PCG (metalFoamBackend::pcg), 1: BiCGStab (::bicgstab).
int inner_solve(cf_context* c, int kind, const double* mean, double target, int maxIter, int ips,
                int order, int useGraph, cf_inner_stats* stats, int stagLimit = STAG_LIMIT,
                int persistMax = 0, int clusterMax = 0)
{
    const double tw0 = wall_now();
    cudaStream_t s = c->stream;
    if (kind == 0 && order > 1)
    {
        if (order > CF_MAX_CHEB) return fail(CF_ERR_INVALID_ARG, "chebyshevOrder too large");
    }
    k_inner_setup<<<1, 32, 0, s>>>(c->d_st, target, maxIter, ips, stagLimit);
    CF_LAUNCH();
    const PcgBufs B = pcg_bufs(c);
    if (kind == 0)
    {
        if (order > 1)
        {
            auto fn = k_pcg_init<true>;
            fn<<<grid_for(c, (const void*)fn, c->n), NT, 0, s>>>(B, mean, c->d_st, c->d_part);
        }
        else
        {
            auto fn = k_pcg_init<false>;
            fn<<<grid_for(c, (const void*)fn, c->n), NT, 0, s>>>(B, mean, c->d_st, c->d_part);
        }
    }
    else
    {
        k_bicg_init<<<grid_for(c, (const void*)k_bicg_init, c->n), NT, 0, s>>>(
            bicg_bufs(c), mean, c->d_st, c->d_part);
    }
    CF_LAUNCH();
    CF_CUDA(cudaEventRecord(c->ev0, s));
    bool persistent = false;
    bool clustered = false;
    if (maxIter > 0)
    {
        // small PCG systems: the whole loop inside one thread-block cluster
        if (useGraph && spmv_default(c) && kind == 0 && clusterMax >= 0 && !c->amgActive)
            CF_TRY(cluster_inner(c, order, clusterMax == 0 ? 16384 : clusterMax, &clustered));
        // opt-in: the whole loop as one cooperative kernel
        if (!clustered && useGraph && spmv_default(c) && !c->amgActive)
            CF_TRY(persistent_inner(c, kind, kind == 0 ? order : 1, persistMax, &persistent));
        if (persistent || clustered)
        {
            c->pendingBodyKernels = 0;
        }
        else if (useGraph)
        {
            cudaGraphExec_t exec;
            int nk = 0;
            CF_TRY(get_graph(c, kind, order, &exec, &nk));
            CF_CUDA(cudaGraphLaunch(exec, s));
            c->pendingBodyKernels = nk;
        }
        else
        {
            // host-synchronised loop: one device->host read per iteration,
            // the reference's command-buffer structure (metalFoamBackend.C:608-716)
            for (int it = 0; it < maxIter; ++it)
            {
                int nk = 0;
                if (kind == 0)
                    CF_TRY(launch_pcg_body(c, order, 0, 0, &nk));
                else
                    CF_TRY(launch_bicg_body(c, 0, 0, &nk));
                CF_CUDA(cudaMemcpyAsync(c->h_st, c->d_st, sizeof(InnerState),
                                        cudaMemcpyDeviceToHost, s));
                CF_CUDA(cudaStreamSynchronize(s));
                if (c->h_st->done) break;
            }
            c->pendingBodyKernels = 0;
        }
    }
    else
    {
        c->pendingBodyKernels = 0;
    }
    CF_CUDA(cudaEventRecord(c->ev1, s));
    k_inner_final<<<1, 32, 0, s>>>(c->d_st);
    CF_LAUNCH();
    CF_CUDA(cudaMemcpyAsync(c->h_st, c->d_st, sizeof(InnerState), cudaMemcpyDeviceToHost, s));
    CF_CUDA(cudaStreamSynchronize(s));
    if (persistent) CF_TRY(persistent_status(c));
    const InnerState& st = *c->h_st;
    if (c->pendingBodyKernels) c->launches += (long long)c->pendingBodyKernels * std::max(st.it, 1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    if (stats)
    {
        stats->nIterations = st.it;
        stats->converged = st.converged;
        stats->singular = st.singular;
        stats->stagnated = st.stagnated;
        stats->finalResSum = st.finalResSum;
        stats->tGpuSeconds = ms * 1e-3;
        stats->tWallSeconds = wall_now() - tw0;
    }
    c->lastInnerKind = kind;
    return CF_OK;
}

int check_ready(cf_context* c)
{
    if (!c) return fail(CF_ERR_INVALID_ARG, "context is NULL");
    if (!c->hasTopo) return fail(CF_ERR_NO_TOPOLOGY, "cf_set_topology has not been called");
    if (!c->hasCoeffs) return fail(CF_ERR_NO_COEFFS, "cf_set_coeffs has not been called");
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return fail(CF_ERR_CUDA, cudaGetErrorString(e));
    return CF_OK;
}

int upload_r64(cf_context* c, const double* r_host)
{
    CF_CUDA(cudaMemcpyAsync(c->d_io64, r_host, sizeof(double) * c->n, cudaMemcpyHostToDevice,
                            c->stream));
    k_gather_f64<<<grid_for(c, (const void*)k_gather_f64, c->n), NT, 0, c->stream>>>(
        c->n, c->d_perm, c->d_io64, c->d_r64);
    CF_LAUNCH();
    return CF_OK;
}

bool check_convergence(double tol, double relTol, double initial, double final_)
{
    // SolverPerformance::checkConvergence
    return (final_ < tol) || (relTol > 1e-20 && final_ < relTol * initial);
}

int fetch_drv(cf_context* c)
{
    CF_CUDA(cudaMemcpyAsync(c->h_drv, c->d_drv, sizeof(DriverState), cudaMemcpyDeviceToHost,
                            c->stream));
    CF_CUDA(cudaStreamSynchronize(c->stream));
    return CF_OK;
}

// metalFoamSolver::solveImpl on the device.  psi_dev / src_dev are in the
// caller's cell order on the device.
int solve_device(cf_context* c, int solver, double* psi_dev, const double* src_dev,
                 const cf_options* o, cf_performance* perf)
{
    const bool bicg = solver == CF_SOLVER_PBICGSTAB;
    const char* name = bicg ? "cudaPBiCGStab" : "cudaPCG";
    cudaStream_t s = c->stream;
    const int n = c->n;
    const DevSell A = sell_of(c);
    std::memset(perf, 0, sizeof(*perf));
    const bool gamg = o->preconditioner == CF_PRECOND_GAMG;
    if (gamg && bicg)
        return fail(CF_ERR_UNSUPPORTED, "the GAMG preconditioner is offered for cudaPCG only");
    // the V-cycle replaces the Chebyshev apply for this solve only
    struct AmgScope
    {
        cf_context* c;
        ~AmgScope() { c->amgActive = false; }
    } amgScope{c};
    CF_CUDA(cudaEventRecord(c->ev2, s));

    // FP32 operator symmetric for PCG, as the reference stages it
    // (metalFoamSolver.C:211-220)
    const int wantSym32 = (!bicg || !c->hasLower) ? 1 : 0;
    if (wantSym32 != c->val32Sym) CF_TRY(stage_vals(c, wantSym32));

    const int gRow = grid_for(c, (const void*)k_gather_f64, n);
    k_gather_f64<<<gRow, NT, 0, s>>>(n, c->d_perm, psi_dev, c->d_psi);
    CF_LAUNCH();
    k_gather_f64<<<gRow, NT, 0, s>>>(n, c->d_perm, src_dev, c->d_b);
    CF_LAUNCH();

    // initial residual, normFactor (metalFoamSolver.C:109-129)
    k_mean_f64<<<grid_for(c, (const void*)k_mean_f64, n), NT, 0, s>>>(
        n, c->d_psi, &c->d_drv->xbar, &c->d_drv->ticket, c->d_part);
    CF_LAUNCH();
    {
        auto fn = k_residual0<MW>;
        fn<<<grid_for(c, (const void*)fn, n), NT, 0, s>>>(A, c->d_diag64, c->d_psi, c->d_b, c->d_u,
                                                         c->d_r64, c->d_drv, c->d_part);
        CF_LAUNCH();
    }
    CF_CUDA(cudaMemcpyAsync(c->d_r0, c->d_r64, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    CF_TRY(fetch_drv(c));
    c->hasResidual = true;
    perf->normFactor = c->h_drv->normFactor;
    perf->initialResidual = c->h_drv->initRes;
    perf->finalResidual = perf->initialResidual;
    perf->chebBeta = 2.0;

    if (o->minIter > 0 ||
        !check_convergence(o->tolerance, o->relTol, perf->initialResidual, perf->finalResidual))
    {
        perf->solved = 1;
        // deflation decision (metalFoamSolver.C:170-209)
        bool deflate = false;
        if (!bicg && o->deflate != CF_DEFLATE_OFF)
        {
            if (o->deflate == CF_DEFLATE_ON)
                deflate = true;
            else
                deflate = (10LL * c->h_drv->nPinned <= (long long)n);
        }
        if (deflate && c->h_drv->signflip) deflate = false;
        perf->deflated = deflate;
        const double tc0 = wall_now();
        CF_TRY(stage_diag32(c, deflate ? 1 : 0));
        if (gamg)
        {
            CF_TRY(amg_prepare(c, o->nCellsInCoarsestLevel, o->profile != 0));
            CF_TRY(amg_stage(c, deflate ? 1 : 0, (float)o->scaleCorrection));
            c->amgActive = true;
        }

        // Chebyshev setup (metalFoamSolver.C:224-249); with GAMG the
        // constants are the smoother's (degree nSweeps)
        const int order = bicg ? 1 : (gamg ? o->nSweeps : o->chebyshevOrder);
        if (order < 1 || order > CF_MAX_CHEB)
            return fail(CF_ERR_INVALID_ARG, "chebyshevOrder must be in [1, 64]");
        if (order > 1)
        {
            auto fn = k_gershgorin<MW>;
            fn<<<grid_for(c, (const void*)fn, n), NT, 0, s>>>(
                A, c->d_eface, c->d_upper, c->d_diag64, c->d_u, deflate ? 1 : 0, order,
                gamg ? o->smootherRatio : o->chebyshevRatio, c->d_chebC, c->d_drv, c->d_part);
            CF_LAUNCH();
        }
        CF_TRY(fetch_drv(c));
        perf->tConvert = wall_now() - tc0;
        if (order > 1) perf->chebBeta = c->h_drv->chebBeta;

        const double target =
            std::max(o->tolerance, o->relTol * perf->initialResidual) * perf->normFactor;
        int totalIter = 0;
        int outer = 0;
        int singular = 0;
        double prevRes = perf->initialResidual;
        for (outer = 0; outer <= o->maxRestarts; ++outer)
        {
            const double* meanp = nullptr;
            if (deflate)
            {
                k_mean_f64<<<grid_for(c, (const void*)k_mean_f64, n), NT, 0, s>>>(
                    n, c->d_r64, &c->d_drv->rmean, &c->d_drv->ticket, c->d_part);
                CF_LAUNCH();
                meanp = &c->d_drv->rmean;
            }
            cf_inner_stats st;
            CF_TRY(inner_solve(c, bicg ? 1 : 0, meanp, target, o->maxIter - totalIter,
                               o->iterationsPerSync, order, o->graph, &st,
                               o->stagnationLimit > 0 ? o->stagnationLimit : STAG_LIMIT,
                               o->persistentMaxCells, o->clusterMaxCells));
            totalIter += st.nIterations;
            perf->tGpu += st.tGpuSeconds;
            perf->tInner += st.tWallSeconds;
            singular = st.singular;
            perf->stagnated = st.stagnated;
            perf->finalResSum32 = st.finalResSum;

            // psi += delta (- mean delta) (metalFoamSolver.C:318-330)
            const double* dmeanp = nullptr;
            if (deflate)
            {
                k_mean_delta<<<grid_for(c, (const void*)k_mean_delta, n), NT, 0, s>>>(
                    n, c->d_D, c->d_st, &c->d_drv->dmean, &c->d_drv->ticket, c->d_part);
                CF_LAUNCH();
                dmeanp = &c->d_drv->dmean;
            }
            k_psi_update<<<grid_for(c, (const void*)k_psi_update, n), NT, 0, s>>>(
                n, c->d_psi, c->d_D, c->d_st, dmeanp);
            CF_LAUNCH();
            // true FP64 residual, constant-mode shift (metalFoamSolver.C:333-365)
            {
                auto fn = k_residual<MW>;
                fn<<<grid_for(c, (const void*)fn, n), NT, 0, s>>>(A, c->d_diag64, c->d_psi,
                                                                 c->d_b, c->d_u, c->d_r64,
                                                                 deflate ? 1 : 0, c->d_drv,
                                                                 c->d_part);
                CF_LAUNCH();
            }
            if (deflate)
            {
                k_cshift<<<grid_for(c, (const void*)k_cshift, n), NT, 0, s>>>(
                    n, c->d_psi, c->d_r64, c->d_u, c->d_drv, c->d_part);
                CF_LAUNCH();
            }
            CF_TRY(fetch_drv(c));
            perf->finalResidual = c->h_drv->finalRes;
            perf->nIterations = totalIter;

            // hybrid polish (metalFoamSolver.C:371-390); chebBeta is kept
            if (deflate && perf->finalResidual > prevRes / 1.5 && !st.singular)
            {
                deflate = false;
                perf->polished = 1;
                CF_TRY(stage_diag32(c, 0));
                if (gamg) CF_TRY(amg_stage(c, 0, (float)o->scaleCorrection));
                if (o->verbose)
                    std::printf("    %s switching to exact operator (polish)\n", name);
            }
            prevRes = perf->finalResidual;
            if (o->verbose)
                std::printf("    %s restart %d: inner=%d fp32ResSum=%g fp64Res=%g%s%s\n", name,
                            outer, st.nIterations, st.finalResSum, perf->finalResidual,
                            st.stagnated ? " (stagnated)" : "", st.singular ? " (breakdown)" : "");
            if (singular) break;
            if (totalIter >= o->maxIter) break;
            if (perf->nIterations >= o->minIter &&
                check_convergence(o->tolerance, o->relTol, perf->initialResidual,
                                  perf->finalResidual))
                break;
        }
        perf->nRestarts = outer;
        perf->singular = singular;
    }
    perf->converged =
        check_convergence(o->tolerance, o->relTol, perf->initialResidual, perf->finalResidual);
    k_l2<<<grid_for(c, (const void*)k_l2, n), NT, 0, s>>>(n, c->d_r64, c->d_b, c->d_drv,
                                                         c->d_part);
    CF_LAUNCH();
    k_scatter_f64<<<gRow, NT, 0, s>>>(n, c->d_perm, c->d_psi, psi_dev);
    CF_LAUNCH();
    CF_CUDA(cudaEventRecord(c->ev3, s));
    CF_TRY(fetch_drv(c));
    perf->residualL2 = c->h_drv->l2b > 0 ? c->h_drv->l2r / c->h_drv->l2b : c->h_drv->l2r;
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, c->ev2, c->ev3);
    perf->tSolve = ms * 1e-3;
    if (o->profile)
        std::printf("    %s profile: cells=%d iters=%d restarts=%d tConvert=%gms tInner=%gms "
                    "tGpu=%gms tSolve=%gms\n",
                    name, n, perf->nIterations, perf->nRestarts, 1000 * perf->tConvert,
                    1000 * perf->tInner, 1000 * perf->tGpu, 1000 * perf->tSolve);
    return CF_OK;
}

int check_options(const cf_options* o)
{
    if (!o) return fail(CF_ERR_INVALID_ARG, "options is NULL");
    if (o->deflate < CF_DEFLATE_AUTO || o->deflate > CF_DEFLATE_OFF)
        return fail(CF_ERR_INVALID_ARG, "deflate must be auto, on or off");
    if (o->maxRestarts < 0) return fail(CF_ERR_INVALID_ARG, "maxRestarts must be >= 0");
    if (!(o->chebyshevRatio > 1.0)) return fail(CF_ERR_INVALID_ARG, "chebyshevRatio must be > 1");
    if (o->preconditioner != CF_PRECOND_CHEBYSHEV && o->preconditioner != CF_PRECOND_GAMG)
        return fail(CF_ERR_INVALID_ARG, "preconditioner must be Chebyshev or GAMG");
    if (o->preconditioner == CF_PRECOND_GAMG &&
        (o->nSweeps < 2 || o->nSweeps > 8 || o->nCellsInCoarsestLevel < 1 ||
         o->nCellsInCoarsestLevel > 128 || !(o->scaleCorrection > 0.0) ||
         !(o->scaleCorrection < 2.0) || !(o->smootherRatio > 1.0)))
        return fail(CF_ERR_INVALID_ARG, "GAMG: nSweeps must be in [2, 8], "
                                        "nCellsInCoarsestLevel in [1, 128], "
                                        "scaleCorrection in (0, 2) and smootherRatio > 1");
    return CF_OK;
}

}  // namespace

// ------------------------------------------------------------------ inner ABI

extern "C" int cf_pcg(cf_context* c, const double* r, double targetResSum, int32_t maxIter,
                      int32_t iterationsPerSync, int32_t chebOrder, double chebBeta,
                      double chebRatio, cf_inner_stats* stats)
{
    CF_TRY(check_ready(c));
    if (!r) return fail(CF_ERR_INVALID_ARG, "r is NULL");
    if (chebOrder > CF_MAX_CHEB) return fail(CF_ERR_INVALID_ARG, "chebOrder too large");
    if (chebOrder > 1)
    {
        float cc[2 * CF_MAX_CHEB];
        cheb_constants(chebOrder, chebBeta, chebRatio, cc);
        CF_CUDA(cudaMemcpyAsync(c->d_chebC, cc, sizeof(float) * 2 * chebOrder,
                                cudaMemcpyHostToDevice, c->stream));
    }
    CF_TRY(upload_r64(c, r));
    return inner_solve(c, 0, nullptr, targetResSum, maxIter, iterationsPerSync,
                       chebOrder > 1 ? chebOrder : 1, 1, stats);
}

extern "C" int cf_bicgstab(cf_context* c, const double* r, double targetResSum, int32_t maxIter,
                           cf_inner_stats* stats)
{
    CF_TRY(check_ready(c));
    if (!r) return fail(CF_ERR_INVALID_ARG, "r is NULL");
    CF_TRY(upload_r64(c, r));
    return inner_solve(c, 1, nullptr, targetResSum, maxIter, 1, 1, 1, stats);
}

extern "C" int cf_delta(cf_context* c, float* delta)
{
    CF_TRY(check_ready(c));
    if (!delta) return fail(CF_ERR_INVALID_ARG, "delta is NULL");
    const int sel = c->h_st->sel;
    k_scatter_f32<<<grid_for(c, (const void*)k_scatter_f32, c->n), NT, 0, c->stream>>>(
        c->n, c->d_perm, c->d_D + (size_t)sel * c->n, c->d_io32);
    CF_LAUNCH();
    CF_CUDA(cudaMemcpyAsync(delta, c->d_io32, sizeof(float) * c->n, cudaMemcpyDeviceToHost,
                            c->stream));
    CF_CUDA(cudaStreamSynchronize(c->stream));
    return CF_OK;
}

// ------------------------------------------------------------------ full solve

extern "C" int cf_solve_device(cf_context* c, int32_t solver, double* psi, const double* source,
                               const cf_options* o, cf_performance* perf)
{
    CF_TRY(check_ready(c));
    CF_TRY(check_options(o));
    if (!psi || !source || !perf) return fail(CF_ERR_INVALID_ARG, "NULL argument");
    if (solver != CF_SOLVER_PCG && solver != CF_SOLVER_PBICGSTAB)
        return fail(CF_ERR_INVALID_ARG, "unknown solver");
    return solve_device(c, solver, psi, source, o, perf);
}

extern "C" int cf_solve(cf_context* c, int32_t solver, double* psi, const double* source,
                        const cf_options* o, cf_performance* perf)
{
    CF_TRY(check_ready(c));
    CF_TRY(check_options(o));
    if (!psi || !source || !perf) return fail(CF_ERR_INVALID_ARG, "NULL argument");
    if (solver != CF_SOLVER_PCG && solver != CF_SOLVER_PBICGSTAB)
        return fail(CF_ERR_INVALID_ARG, "unknown solver");
    CF_CUDA(cudaMemcpyAsync(c->d_io64, psi, sizeof(double) * c->n, cudaMemcpyHostToDevice,
                            c->stream));
    CF_CUDA(cudaMemcpyAsync(c->d_io64b, source, sizeof(double) * c->n, cudaMemcpyHostToDevice,
                            c->stream));
    CF_TRY(solve_device(c, solver, c->d_io64, c->d_io64b, o, perf));
    CF_CUDA(cudaMemcpyAsync(psi, c->d_io64, sizeof(double) * c->n, cudaMemcpyDeviceToHost,
                            c->stream));
    CF_CUDA(cudaStreamSynchronize(c->stream));
    return CF_OK;
}

extern "C" int cf_residual(cf_context* c, int32_t which, double* r)
{
    CF_TRY(check_ready(c));
    if (!r || (which != 0 && which != 1)) return fail(CF_ERR_INVALID_ARG, "bad arguments");
    if (!c->hasResidual) return fail(CF_ERR_INVALID_ARG, "no solve has run on this context");
    const int n = c->n;
    k_scatter_f64<<<grid_for(c, (const void*)k_scatter_f64, n), NT, 0, c->stream>>>(
        n, c->d_perm, which == 0 ? c->d_r0 : c->d_r64, c->d_io64b);
    CF_LAUNCH();
    CF_CUDA(cudaMemcpyAsync(r, c->d_io64b, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
    CF_CUDA(cudaStreamSynchronize(c->stream));
    return CF_OK;
}

// ------------------------------------------------------------------ operators

extern "C" int cf_amul(cf_context* c, const double* x, double* y, int32_t transpose)
{
    CF_TRY(check_ready(c));
    if (!x || !y) return fail(CF_ERR_INVALID_ARG, "NULL argument");
    const int n = c->n;
    cudaStream_t s = c->stream;
    CF_CUDA(cudaMemcpyAsync(c->d_io64, x, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    k_gather_f64<<<grid_for(c, (const void*)k_gather_f64, n), NT, 0, s>>>(n, c->d_perm,
                                                                          c->d_io64, c->d_psi);
    CF_LAUNCH();
    auto fn = k_amul64<MW>;
    fn<<<grid_for(c, (const void*)fn, n), NT, 0, s>>>(sell_of(c),
                                                     transpose ? c->d_valT64 : c->d_val64,
                                                     c->d_diag64, c->d_psi, c->d_r64);
    CF_LAUNCH();
    k_scatter_f64<<<grid_for(c, (const void*)k_scatter_f64, n), NT, 0, s>>>(n, c->d_perm,
                                                                           c->d_r64, c->d_io64);
    CF_LAUNCH();
    CF_CUDA(cudaMemcpyAsync(y, c->d_io64, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
    CF_CUDA(cudaStreamSynchronize(s));
    return CF_OK;
}

extern "C" int cf_spmv32(cf_context* c, const float* x, const float* w, float* y, double* dot)
{
    CF_TRY(check_ready(c));
    if (!x || !y) return fail(CF_ERR_INVALID_ARG, "NULL argument");
    const int n = c->n;
    cudaStream_t s = c->stream;
    const int g = grid_for(c, (const void*)k_gather_f32, n);
    CF_CUDA(cudaMemcpyAsync(c->d_io32, x, sizeof(float) * n, cudaMemcpyHostToDevice, s));
    k_gather_f32<<<g, NT, 0, s>>>(n, c->d_perm, c->d_io32, c->d_Z0);
    CF_LAUNCH();
    if (w)
    {
        CF_CUDA(cudaMemcpyAsync(c->d_io32, w, sizeof(float) * n, cudaMemcpyHostToDevice, s));
        k_gather_f32<<<g, NT, 0, s>>>(n, c->d_perm, c->d_io32, c->d_Z1);
        CF_LAUNCH();
    }
    if (!spmv_default(c))
    {
        CF_TRY(launch_spmv32_v(c, c->d_diag32, c->d_Z0, w ? c->d_Z1 : nullptr, c->d_W1,
                               c->d_scratch64));
    }
    else
    {
        const DevSell A = sell_of(c);
        auto fn = spmv32_kernel(A);
        fn<<<grid_for(c, (const void*)fn, n), NT, 0, s>>>(A, c->d_diag32, c->d_Z0,
                                                         w ? c->d_Z1 : nullptr, c->d_W1,
                                                         c->d_scratch64, &c->d_drv->ticket,
                                                         c->d_part);
        CF_LAUNCH();
    }
    k_scatter_f32<<<g, NT, 0, s>>>(n, c->d_perm, c->d_W1, c->d_io32);
    CF_LAUNCH();
    CF_CUDA(cudaMemcpyAsync(y, c->d_io32, sizeof(float) * n, cudaMemcpyDeviceToHost, s));
    double h = 0.0;
    CF_CUDA(cudaMemcpyAsync(&h, c->d_scratch64, sizeof(double), cudaMemcpyDeviceToHost, s));
    CF_CUDA(cudaStreamSynchronize(s));
    if (dot) *dot = w ? h : 0.0;
    return CF_OK;
}

extern "C" int cf_cheb_apply(cf_context* c, const float* r, float* z, int32_t order, double beta,
                             double ratio)
{
    CF_TRY(check_ready(c));
    if (!r || !z) return fail(CF_ERR_INVALID_ARG, "NULL argument");
    if (order < 1 || order > CF_MAX_CHEB) return fail(CF_ERR_INVALID_ARG, "order out of range");
    const int n = c->n;
    cudaStream_t s = c->stream;
    float cc[2 * CF_MAX_CHEB];
    cheb_constants(order, beta, ratio, cc);
    CF_CUDA(cudaMemcpyAsync(c->d_chebC, cc, sizeof(float) * std::max(2 * order, 2),
                            cudaMemcpyHostToDevice, s));
    const int g = grid_for(c, (const void*)k_gather_f32, n);
    CF_CUDA(cudaMemcpyAsync(c->d_io32, r, sizeof(float) * n, cudaMemcpyHostToDevice, s));
    k_gather_f32<<<g, NT, 0, s>>>(n, c->d_perm, c->d_io32, c->d_rA);
    CF_LAUNCH();
    k_cheb_init<<<g, NT, 0, s>>>(n, c->d_rA, c->d_rD32, c->d_chebC, c->d_W0);
    CF_LAUNCH();
    // a fresh state so the step kernels run (done = 0)
    k_inner_setup<<<1, 32, 0, s>>>(c->d_st, 0.0, 1, 1);
    CF_LAUNCH();
    const DevSell A = sell_of(c);
    const PcgBufs B = pcg_bufs(c);
    const float* out = c->d_W0;
    float* Z[2] = {c->d_Z0, c->d_Z1};
    for (int j = 1; j < order; ++j)
    {
        const float* zin = (j == 1) ? B.W0 : Z[chebz(j - 1)];
        const float* win = (j == 1) ? B.W0 : B.W1;
        if (!spmv_default(c))
        {
            CF_TRY(launch_cheb_step_v(c, false, B, zin, win, B.W1, Z[chebz(j)], j));
        }
        else
        {
            auto fn = cheb_step_kernel<false>(A);
            fn<<<rows_grid(n), NT, 0, s>>>(A, B, zin, win, B.W1, Z[chebz(j)], j, c->d_st,
                                           c->d_part);
            CF_LAUNCH();
        }
        out = Z[chebz(j)];
    }
    k_scatter_f32<<<g, NT, 0, s>>>(n, c->d_perm, out, c->d_io32);
    CF_LAUNCH();
    CF_CUDA(cudaMemcpyAsync(z, c->d_io32, sizeof(float) * n, cudaMemcpyDeviceToHost, s));
    CF_CUDA(cudaStreamSynchronize(s));
    return CF_OK;
}

// ------------------------------------------------------------------ measurement

extern "C" int cf_time_kernel(cf_context* c, int32_t which, int32_t reps, double* msPerLaunch)
{
    CF_TRY(check_ready(c));
    if (!msPerLaunch || reps <= 0) return fail(CF_ERR_INVALID_ARG, "bad arguments");
    const int n = c->n;
    cudaStream_t s = c->stream;
    const DevSell A = sell_of(c);
    const PcgBufs B = pcg_bufs(c);
    // operands with finite values and a live (not done) state
    float cc[2 * 8];
    cheb_constants(8, 2.0, 30.0, cc);
    CF_CUDA(cudaMemcpyAsync(c->d_chebC, cc, sizeof(cc), cudaMemcpyHostToDevice, s));
    k_inner_setup<<<1, 32, 0, s>>>(c->d_st, 0.0, 1 << 30, 1);
    CF_LAUNCH();
    const int g1 = grid_for(c, (const void*)k_cheb_init, n);
    k_cheb_init<<<g1, NT, 0, s>>>(n, B.rA, B.rD, c->d_chebC, B.W0);
    CF_LAUNCH();
    k_cheb_init<<<g1, NT, 0, s>>>(n, B.rA, B.rD, c->d_chebC, B.Z0);
    CF_LAUNCH();
    k_cheb_init<<<g1, NT, 0, s>>>(n, B.rA, B.rD, c->d_chebC, B.W1);
    CF_LAUNCH();
    CF_CUDA(cudaMemsetAsync(c->d_P, 0, sizeof(float) * 2 * (size_t)n, s));
    if (which == CF_KERNEL_SPMV32_COLD)
    {
        // every launch starts from a cold L2: 256 MB (twice the L2) READ
        // between launches -- a read leaves clean lines, so no write-back of
        // the flush competes with the timed SpMV -- only the SpMV bracketed
        // by events
        const size_t flushBytes = (size_t)256 << 20;
        void* flush = nullptr;
        if (cudaMalloc(&flush, flushBytes) != cudaSuccess)
        {
            cudaGetLastError();
            return fail(CF_ERR_CUDA, "cf_time_kernel: no room for the L2 flush buffer");
        }
        double total = 0.0;
        int rc = CF_OK;
        auto fn = spmv32_kernel(A);
        const int g = grid_for(c, (const void*)fn, n);
        cudaMemsetAsync(flush, 0, flushBytes, s);
        const int gf = grid_for(c, (const void*)k_read_flush, (long long)(flushBytes / 16));
        for (int i = 0; i < reps && rc == CF_OK; ++i)
        {
            k_read_flush<<<gf, NT, 0, s>>>(reinterpret_cast<const float4*>(flush),
                                           (long long)(flushBytes / 16), c->d_scratch64 + 1);
            cudaEventRecord(c->ev0, s);
            fn<<<g, NT, 0, s>>>(A, B.diag, B.Z0, B.W0, B.Z1, c->d_scratch64, &c->d_drv->ticket,
                                c->d_part);
            cudaEventRecord(c->ev1, s);
            const cudaError_t e = cudaEventSynchronize(c->ev1);
            if (e != cudaSuccess)
            {
                rc = fail(CF_ERR_CUDA, cudaGetErrorString(e));
                break;
            }
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, c->ev0, c->ev1);
            total += ms;
            c->launches++;
        }
        cudaFree(flush);
        if (rc != CF_OK) return rc;
        *msPerLaunch = total / reps;
        return CF_OK;
    }
    if (which == CF_KERNEL_CHEB_STEP_INNER)
    {
        // full PCG iterations (Chebyshev 8, p-update SpMV, update) launched
        // one by one from the solve's own inner right-hand side, the 7 steps
        // of each iteration bracketed by events
        k_inner_setup<<<1, 32, 0, s>>>(c->d_st, 0.0, 1 << 30, 1, 1 << 30);
        CF_LAUNCH();
        k_pcg_init<true><<<grid_for(c, (const void*)k_pcg_init<true>, n), NT, 0, s>>>(
            B, nullptr, c->d_st, c->d_part);
        CF_LAUNCH();
        const int steps = 7 * reps;
        std::vector<cudaEvent_t> ev(2 * (size_t)steps, nullptr);
        for (auto& e : ev)
            if (cudaEventCreate(&e) != cudaSuccess)
            {
                for (auto& f : ev)
                    if (f) cudaEventDestroy(f);
                return fail(CF_ERR_CUDA, "cudaEventCreate");
            }
        int k = 0;
        int rc = CF_OK;
        float* Z[2] = {B.Z0, B.Z1};
        for (int it = 0; it < reps && rc == CF_OK; ++it)
        {
            for (int j = 1; j < 8 && rc == CF_OK; ++j)
            {
                const float* zin = (j == 1) ? B.W0 : Z[chebz(j - 1)];
                const float* win = (j == 1) ? B.W0 : B.W1;
                cudaEventRecord(ev[2 * k], s);
                {
                    auto fn = j == 7 ? cheb_step_kernel<true>(A) : cheb_step_kernel<false>(A);
                    fn<<<j == 7 ? grid_for(c, (const void*)fn, n) : rows_grid(n), NT, 0, s>>>(
                        A, B, zin, win, B.W1, Z[chebz(j)], j, c->d_st, c->d_part);
                }
                cudaEventRecord(ev[2 * k + 1], s);
                ++k;
                const cudaError_t e = cudaGetLastError();
                if (e != cudaSuccess) rc = fail(CF_ERR_CUDA, cudaGetErrorString(e));
            }
            if (rc != CF_OK) break;
            {
                auto fp = pcg_p_spmv_kernel(A);
                fp<<<grid_for(c, (const void*)fp, n), NT, 0, s>>>(A, B, Z[chebz(7)], c->d_st,
                                                                 c->d_part);
            }
            k_pcg_update<true><<<grid_for(c, (const void*)k_pcg_update<true>, n), NT, 0, s>>>(
                B, c->d_st, c->d_part, 0, 0);
        }
        double total = 0.0;
        if (rc == CF_OK && cudaStreamSynchronize(s) == cudaSuccess)
        {
            for (int i = 0; i < k; ++i)
            {
                float ms = 0.0f;
                cudaEventElapsedTime(&ms, ev[2 * i], ev[2 * i + 1]);
                total += ms;
            }
            c->launches += (long long)reps * 9;
        }
        else if (rc == CF_OK)
        {
            rc = fail(CF_ERR_CUDA, "cudaStreamSynchronize");
        }
        for (auto& e : ev) cudaEventDestroy(e);
        if (rc != CF_OK) return rc;
        // every timed step must have run its rows: a state that ended early
        // (an inner right-hand side that is zero, as before any solve) would
        // time kernels that return at once
        CF_CUDA(cudaMemcpy(c->h_st, c->d_st, sizeof(InnerState), cudaMemcpyDeviceToHost));
        if (c->h_st->done)
            return fail(CF_ERR_INVALID_ARG,
                        "cf_time_kernel(CHEB_STEP_INNER): the inner state ended before the timed "
                        "iterations (zero inner right-hand side: run a solve first)");
        *msPerLaunch = total / steps;
        return CF_OK;
    }
    auto launch = [&]() -> int {
        switch (which)
        {
            case CF_KERNEL_CHEB_STEP:
            {
                if (!spmv_default(c))
                    return launch_cheb_step_v(c, false, B, B.Z0, B.W1, B.W1, B.Z1, 2);
                auto fn = cheb_step_kernel<false>(A);
                fn<<<rows_grid(n), NT, 0, s>>>(A, B, B.Z0, B.W1, B.W1, B.Z1, 2, c->d_st,
                                               c->d_part);
                break;
            }
            case CF_KERNEL_SPMV32:
            {
                if (!spmv_default(c))
                    return launch_spmv32_v(c, B.diag, B.Z0, B.W0, B.Z1, c->d_scratch64);
                auto fn = spmv32_kernel(A);
                fn<<<grid_for(c, (const void*)fn, n), NT, 0, s>>>(A, B.diag, B.Z0, B.W0, B.Z1,
                                                                 c->d_scratch64,
                                                                 &c->d_drv->ticket, c->d_part);
                break;
            }
            case CF_KERNEL_PCG_P_SPMV:
            {
                if (!spmv_default(c)) return launch_pcg_p_spmv_v(c, B, B.Z0);
                auto fn = pcg_p_spmv_kernel(A);
                fn<<<grid_for(c, (const void*)fn, n), NT, 0, s>>>(A, B, B.Z0, c->d_st, c->d_part);
                break;
            }
            case CF_KERNEL_PCG_UPDATE:
            {
                auto fn = k_pcg_update<true>;
                fn<<<grid_for(c, (const void*)fn, n), NT, 0, s>>>(B, c->d_st, c->d_part, 0, 0);
                break;
            }
            case CF_KERNEL_AMUL64:
            {
                auto fn = k_amul64<MW>;
                fn<<<grid_for(c, (const void*)fn, n), NT, 0, s>>>(A, c->d_val64, c->d_diag64,
                                                                 c->d_psi, c->d_r64);
                break;
            }
            default:
                return fail(CF_ERR_INVALID_ARG, "unknown kernel id");
        }
        CF_LAUNCH();
        return CF_OK;
    };
    CF_TRY(launch());  // warm
    CF_CUDA(cudaEventRecord(c->ev0, s));
    for (int i = 0; i < reps; ++i) CF_TRY(launch());
    CF_CUDA(cudaEventRecord(c->ev1, s));
    CF_CUDA(cudaEventSynchronize(c->ev1));
    float ms = 0.0f;
    CF_CUDA(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    *msPerLaunch = (double)ms / reps;
    return CF_OK;
}
