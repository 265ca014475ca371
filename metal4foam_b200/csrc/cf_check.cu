// cf_check.cu -- one launch of a fused inner-iteration kernel on
// caller-supplied vectors and scalars (cf_inner_step).
//
// The solver's kernels fuse several of the reference's kernels each
// (metalFoamKernels.metal:64-276,372-458): the p-update into the SpMV's
// gathers, the solution/residual update with the next preconditioner apply,
// the BiCGStab emul/p/s updates into the two SpMVs.  A solve-level test only
// sees whether the iteration still converges; this entry point lets a test
// run one fused kernel exactly as the inner loop launches it (same kernel,
// same launch shape, same buffers) and compare every vector it writes with
// the reference's unfused kernel sequence, and every reduction it folds with
// an FP64 sum of the same products.
//
// Vectors come in the caller's cell order, are gathered into the context's
// internal order (the RCM relabelling), and go back the same way.  The
// kernel reads the solver scalars (alpha, beta, omega) from the inner state,
// as it does inside an iteration; they are written there first, rounded as
// the loop rounds them (FP64 state, rounded to FP32 by the kernel).
#include "cudafoam.h"
#include "cf_host.hpp"

#include <cstring>
#include <string>

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

// host vector (caller's order) -> device vector (internal order)
int put(cf_context* c, const float* h, float* d, const char* name)
{
    if (!h) return fail(CF_ERR_INVALID_ARG, std::string("cf_inner_step: input ") + name + " is NULL");
    CF_CUDA(cudaMemcpyAsync(c->d_io32, h, sizeof(float) * c->n, cudaMemcpyHostToDevice, c->stream));
    k_gather_f32<<<grid_for(c, (const void*)k_gather_f32, c->n), NT, 0, c->stream>>>(
        c->n, c->d_perm, c->d_io32, d);
    CF_LAUNCH();
    return CF_OK;
}

// device vector (internal order) -> host vector (caller's order); NULL h: skipped
int get(cf_context* c, const float* d, float* h)
{
    if (!h) return CF_OK;
    k_scatter_f32<<<grid_for(c, (const void*)k_scatter_f32, c->n), NT, 0, c->stream>>>(
        c->n, c->d_perm, d, c->d_io32);
    CF_LAUNCH();
    CF_CUDA(cudaMemcpyAsync(h, c->d_io32, sizeof(float) * c->n, cudaMemcpyDeviceToHost, c->stream));
    return CF_OK;
}

// the state of iteration 0 of a live inner solve: parity 0 writes P[0..n)
// and reads the "previous" direction from P[n..2n); correction buffers
// cur = 0, nxt = 1; nothing converged, no early exit
InnerState fresh_state(const cf_step_io* io)
{
    InnerState st;
    std::memset(&st, 0, sizeof(st));
    st.alpha = io->alpha;
    st.beta = io->beta;
    st.omega = io->omega;
    st.wArA = 1.0;        // previous wA.rA, so the Jacobi update's beta is finite
    st.rA0rA = 1.0;       // a finite rA0.rA (the BiCGStab breakdown test reads it)
    st.bestRes = 1.0e300;
    st.target = -1.0;     // never reached: no convergence or early exit inside the step
    st.maxIter = 1 << 30;
    st.ips = 1;
    st.stagLimit = 1 << 30;
    st.cur = 0;
    st.best = 0;
    st.nxt = 1;
    return st;
}

}  // namespace

extern "C" int cf_inner_step(cf_context* c, int32_t step, cf_step_io* io)
{
    if (!c || !io) return fail(CF_ERR_INVALID_ARG, "cf_inner_step: NULL argument");
    if (!c->hasTopo) return fail(CF_ERR_NO_TOPOLOGY, "cf_set_topology has not been called");
    if (!c->hasCoeffs) return fail(CF_ERR_NO_COEFFS, "cf_set_coeffs has not been called");
    CF_CUDA(cudaSetDevice(c->device));
    const int n = c->n;
    if (n <= 0) return fail(CF_ERR_INVALID_ARG, "cf_inner_step: empty mesh");
    cudaStream_t s = c->stream;
    const DevSell A = sell_of(c);
    const PcgBufs B = pcg_bufs(c);
    const BicgBufs Bb = bicg_bufs(c);
    const bool cheb = io->chebOrder > 1;
    if ((step == CF_STEP_CHEB || (step == CF_STEP_PCG_UPDATE && cheb)) &&
        (io->chebOrder < 2 || io->chebOrder > CF_MAX_CHEB))
        return fail(CF_ERR_INVALID_ARG, "cf_inner_step: chebOrder must be in [2, 64]");
    if (step == CF_STEP_CHEB && (io->chebStep < 1 || io->chebStep >= io->chebOrder))
        return fail(CF_ERR_INVALID_ARG, "cf_inner_step: chebStep must be in [1, chebOrder)");
    if (cheb)
    {
        float cc[2 * CF_MAX_CHEB] = {0.0f};
        cheb_constants(io->chebOrder, io->chebBeta, io->chebRatio, cc);
        CF_CUDA(cudaMemcpyAsync(c->d_chebC, cc, sizeof(cc), cudaMemcpyHostToDevice, s));
    }
    const InnerState st0 = fresh_state(io);
    *c->h_st = st0;
    CF_CUDA(cudaMemcpyAsync(c->d_st, c->h_st, sizeof(InnerState), cudaMemcpyHostToDevice, s));
    float* Pn = B.P;              // parity 0: this iteration's direction
    float* Pold = B.P + n;        // parity 1: the previous iteration's
    float* D0 = B.D;
    float* D1 = B.D + n;
    const bool dflt = spmv_default(c);
    switch (step)
    {
        case CF_STEP_CHEB:
        {
            // zin = Z0, win = W0 -> wout = W1, zout = Z1 (the loop's buffers
            // rotate the same way); rA and rD as staged
            CF_TRY(put(c, io->zIn, B.Z0, "zIn"));
            CF_TRY(put(c, io->wIn, B.W0, "wIn"));
            CF_TRY(put(c, io->rA, B.rA, "rA"));
            const bool last = io->chebStep == io->chebOrder - 1;
            if (!dflt)
            {
                CF_TRY(launch_cheb_step_v(c, last, B, B.Z0, B.W0, B.W1, B.Z1, io->chebStep));
            }
            else if (last)
            {
                auto fn = cheb_step_kernel<true>(A);
                fn<<<grid_for(c, (const void*)fn, n), NT, 0, s>>>(A, B, B.Z0, B.W0, B.W1, B.Z1,
                                                                 io->chebStep, c->d_st, c->d_part);
                CF_LAUNCH();
            }
            else
            {
                auto fn = cheb_step_kernel<false>(A);
                fn<<<rows_grid(n), NT, 0, s>>>(A, B, B.Z0, B.W0, B.W1, B.Z1, io->chebStep,
                                               c->d_st, c->d_part);
                CF_LAUNCH();
            }
            CF_TRY(get(c, B.W1, io->wOut));
            CF_TRY(get(c, B.Z1, io->zOut));
            break;
        }
        case CF_STEP_PCG_P_SPMV:
        {
            CF_TRY(put(c, io->wA, B.W0, "wA"));
            CF_TRY(put(c, io->pOld, Pold, "pOld"));
            if (!dflt)
            {
                CF_TRY(launch_pcg_p_spmv_v(c, B, B.W0));
            }
            else
            {
                auto fn = pcg_p_spmv_kernel(A);
                fn<<<grid_for(c, (const void*)fn, n), NT, 0, s>>>(A, B, B.W0, c->d_st, c->d_part);
                CF_LAUNCH();
            }
            CF_TRY(get(c, Pn, io->p));
            CF_TRY(get(c, B.Q, io->q));
            break;
        }
        case CF_STEP_PCG_UPDATE:
        {
            CF_TRY(put(c, io->delta, D0, "delta"));
            CF_TRY(put(c, io->p, Pn, "p"));
            CF_TRY(put(c, io->rA, B.rA, "rA"));
            CF_TRY(put(c, io->q, B.Q, "q"));
            if (cheb)
            {
                auto fn = k_pcg_update<true>;
                fn<<<grid_for(c, (const void*)fn, n), NT, 0, s>>>(B, c->d_st, c->d_part, 0, 0);
            }
            else
            {
                auto fn = k_pcg_update<false>;
                fn<<<grid_for(c, (const void*)fn, n), NT, 0, s>>>(B, c->d_st, c->d_part, 0, 0);
            }
            CF_LAUNCH();
            CF_TRY(get(c, D1, io->deltaNext));
            CF_TRY(get(c, B.rA, io->rAOut));
            CF_TRY(get(c, B.W0, io->wAOut));
            break;
        }
        case CF_STEP_BICG_AB:
        {
            CF_TRY(put(c, io->rA, Bb.rA, "rA"));
            CF_TRY(put(c, io->pOld, Pold, "pOld"));
            CF_TRY(put(c, io->AyAOld, Bb.AyA + n, "AyAOld"));
            CF_TRY(put(c, io->rA0, Bb.rA0, "rA0"));
            if (!dflt)
            {
                CF_TRY(launch_bicg_ab_v(c, Bb));
            }
            else
            {
                auto fn = bicg_ab_kernel(A);
                fn<<<grid_for(c, (const void*)fn, n), NT, 0, s>>>(A, Bb, c->d_st, c->d_part);
                CF_LAUNCH();
            }
            CF_TRY(get(c, Pn, io->p));
            CF_TRY(get(c, Bb.yA, io->yA));
            CF_TRY(get(c, Bb.AyA, io->AyA));
            break;
        }
        case CF_STEP_BICG_CD:
        {
            CF_TRY(put(c, io->rA, Bb.rA, "rA"));
            CF_TRY(put(c, io->AyA, Bb.AyA, "AyA"));
            if (!dflt)
            {
                CF_TRY(launch_bicg_cd_v(c, Bb, 0, 0));
            }
            else
            {
                auto fn = bicg_cd_kernel(A);
                fn<<<grid_for(c, (const void*)fn, n), NT, 0, s>>>(A, Bb, c->d_st, c->d_part, 0, 0);
                CF_LAUNCH();
            }
            CF_TRY(get(c, Bb.sA, io->sA));
            CF_TRY(get(c, Bb.zA, io->zA));
            CF_TRY(get(c, Bb.tA, io->tA));
            break;
        }
        case CF_STEP_BICG_E:
        {
            CF_TRY(put(c, io->delta, D0, "delta"));
            CF_TRY(put(c, io->yA, Bb.yA, "yA"));
            CF_TRY(put(c, io->zA, Bb.zA, "zA"));
            CF_TRY(put(c, io->sA, Bb.sA, "sA"));
            CF_TRY(put(c, io->tA, Bb.tA, "tA"));
            CF_TRY(put(c, io->rA0, Bb.rA0, "rA0"));
            k_bicg_e<<<grid_for(c, (const void*)k_bicg_e, n), NT, 0, s>>>(Bb, c->d_st, c->d_part,
                                                                          0, 0);
            CF_LAUNCH();
            CF_TRY(get(c, D1, io->deltaNext));
            CF_TRY(get(c, Bb.rA, io->rAOut));
            break;
        }
        default:
            return fail(CF_ERR_INVALID_ARG, "cf_inner_step: unknown step " + std::to_string(step));
    }
    CF_CUDA(cudaMemcpyAsync(c->h_st, c->d_st, sizeof(InnerState), cudaMemcpyDeviceToHost, s));
    CF_CUDA(cudaStreamSynchronize(s));
    const InnerState& st = *c->h_st;
    io->sums[0] = io->sums[1] = io->sums[2] = 0.0;
    switch (step)
    {
        case CF_STEP_CHEB:   // z.r, formed by the last step only
            io->sums[0] = io->chebStep == io->chebOrder - 1 ? st.wArA : 0.0;
            break;
        case CF_STEP_PCG_P_SPMV: io->sums[0] = st.wApA; break;
        case CF_STEP_PCG_UPDATE:
            io->sums[0] = st.res;                          // sum |rA|
            io->sums[1] = cheb ? 0.0 : st.wArA;            // Jacobi: wA.rA
            break;
        case CF_STEP_BICG_AB: io->sums[0] = st.rA0AyA; break;
        case CF_STEP_BICG_CD:
            io->sums[0] = st.resS;                         // sum |s|
            io->sums[1] = st.tAsA;
            io->sums[2] = st.tAtA;
            break;
        case CF_STEP_BICG_E:
            io->sums[0] = st.res;                          // sum |rA|
            io->sums[1] = st.rA0rA;
            break;
    }
    return CF_OK;
}
