// cf_adjoint.cu -- adjoint of the solve x = A^{-1} b (no counterpart in the
// reference; the design's differentiation row).
//
// For a loss L(x): lambda = A^{-T} dL/dx, then
//   dL/db        =  lambda
//   dL/ddiag[i]  = -lambda[i] x[i]
//   dL/dupper[f] = -lambda[l(f)] x[u(f)]     (upper[f] = A[l(f), u(f)])
//   dL/dlower[f] = -lambda[u(f)] x[l(f)]     (lower[f] = A[u(f), l(f)])
// A^T in LDU form is the same matrix with upper and lower exchanged, so the
// transpose solve reuses every kernel of the forward solve on restaged
// values (cf_set_transpose); the gradients come from one face-parallel pass.
#include "cudafoam.h"
#include "cf_host.hpp"

#include <algorithm>
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

// One thread per face (grid-stride), then one per cell; lambda and x in the
// caller's cell order, faces in LDU order.
__global__ void k_face_gradients(int n, int nf, const int* __restrict__ low,
                                 const int* __restrict__ upp, const double* __restrict__ lam,
                                 const double* __restrict__ x, double* __restrict__ dU,
                                 double* __restrict__ dL, double* __restrict__ dD)
{
    const int stride = gridDim.x * blockDim.x;
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < nf; f += stride)
    {
        const int l = low[f];
        const int u = upp[f];
        dU[f] = -__dmul_rn(lam[l], x[u]);
        dL[f] = -__dmul_rn(lam[u], x[l]);
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        dD[i] = -__dmul_rn(lam[i], x[i]);
}

// Source transfer for the transpose solve.  With u = A^T 1 (row sums of the
// staged A^T), A^T 1 = u gives A^{-T} u = 1, so for any c
//   lambda = A^{-T} (g - c u) + c 1.
// c = sum(g)/sum(u) makes the shifted source sum to zero: the consistent,
// pressure-like right-hand side the deflated driver resolves (a source
// with a nonzero sum on a singly pinned Neumann matrix answers with a
// point sink at the pinned cell, which the zero-mean inner solves cannot
// represent).  out[2] = c.
__global__ void __launch_bounds__(NT) k_source_sums(int n, const double* __restrict__ g,
                                                    const double* __restrict__ u, double* out,
                                                    unsigned int* ticket, double* part)
{
    double acc[2] = {0.0, 0.0};
    for (int i = blockIdx.x * NT + threadIdx.x; i < n; i += gridDim.x * NT)
    {
        acc[0] += g[i];
        acc[1] += u[i];
    }
    if (grid_sum<2>(acc, part, ticket) && threadIdx.x == 0)
    {
        out[0] = acc[0];
        out[1] = acc[1];
        out[2] = fabs(acc[1]) > VSMALL ? acc[0] / acc[1] : 0.0;
    }
}

// gs[perm[r]] = g[perm[r]] - c u[r]  (g, gs in the caller's order, u internal)
__global__ void k_shift_source(int n, const int* __restrict__ perm, const double* __restrict__ g,
                               const double* __restrict__ u, const double* cptr,
                               double* __restrict__ gs)
{
    const double c = cptr[2];
    for (int r = blockIdx.x * NT + threadIdx.x; r < n; r += gridDim.x * NT)
    {
        const int i = perm[r];
        gs[i] = __dsub_rn(g[i], __dmul_rn(c, u[r]));
    }
}

__global__ void k_add_const(int n, double* __restrict__ x, const double* cptr)
{
    const double c = cptr[2];
    for (int i = blockIdx.x * NT + threadIdx.x; i < n; i += gridDim.x * NT)
        x[i] = __dadd_rn(x[i], c);
}

// Transpose solve with the source transfer; g and lambda in the caller's
// order on the device, gs a caller-order scratch vector.
int adjoint_solve(cf_context* c, int32_t solver, const double* g, double* gs, double* lambda,
                  const cf_options* opts, cf_performance* perf)
{
    const int n = c->n;
    cudaStream_t s = c->stream;
    CF_CUDA(cudaMemsetAsync(lambda, 0, sizeof(double) * n, s));
    CF_TRY(cf_set_transpose(c, 1));
    k_source_sums<<<grid_for(c, (const void*)k_source_sums, n), NT, 0, s>>>(
        n, g, c->d_u, c->d_scratch64, &c->d_drv->ticket, c->d_part);
    CF_LAUNCH();
    k_shift_source<<<grid_for(c, (const void*)k_shift_source, n), NT, 0, s>>>(
        n, c->d_perm, g, c->d_u, c->d_scratch64, gs);
    CF_LAUNCH();
    int rc = cf_solve_device(c, solver, lambda, gs, opts, perf);
    int rc2 = cf_set_transpose(c, 0);
    if (rc != CF_OK) return rc;
    if (rc2 != CF_OK) return rc2;
    k_add_const<<<grid_for(c, (const void*)k_add_const, n), NT, 0, s>>>(n, lambda,
                                                                       c->d_scratch64);
    CF_LAUNCH();
    return CF_OK;
}

int check_ctx(cf_context* c)
{
    if (!c) return fail(CF_ERR_INVALID_ARG, "context is NULL");
    if (!c->hasTopo) return fail(CF_ERR_NO_TOPOLOGY, "cf_set_topology has not been called");
    if (!c->hasCoeffs) return fail(CF_ERR_NO_COEFFS, "cf_set_coeffs has not been called");
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return fail(CF_ERR_CUDA, cudaGetErrorString(e));
    return CF_OK;
}

int launch_gradients(cf_context* c, const double* lam, const double* x, double* dU, double* dL,
                     double* dD)
{
    const long long work = std::max((long long)c->nf, (long long)c->n);
    const int g = grid_for(c, (const void*)k_face_gradients, work);
    k_face_gradients<<<g, NT, 0, c->stream>>>(c->n, c->nf, c->d_low, c->d_upp, lam, x, dU, dL,
                                              dD);
    CF_LAUNCH();
    return CF_OK;
}

}  // namespace

extern "C" int cf_set_transpose(cf_context* c, int32_t on)
{
    CF_TRY(check_ctx(c));
    const bool t = on != 0;
    if (t == c->transposed) return CF_OK;
    c->transposed = t;
    CF_TRY(stage_vals(c, c->val32Sym));
    CF_TRY(stage_rowsums(c));
    CF_TRY(stage_diag32(c, 0));
    return CF_OK;
}

extern "C" int cf_face_gradients_device(cf_context* c, const double* lambda, const double* x,
                                        double* dUpper, double* dLower, double* dDiag)
{
    CF_TRY(check_ctx(c));
    if (!lambda || !x || !dUpper || !dLower || !dDiag)
        return fail(CF_ERR_INVALID_ARG, "NULL argument");
    return launch_gradients(c, lambda, x, dUpper, dLower, dDiag);
}

extern "C" int cf_face_gradients(cf_context* c, const double* lambda, const double* x,
                                 double* dUpper, double* dLower, double* dDiag)
{
    CF_TRY(check_ctx(c));
    if (!lambda || !x || !dUpper || !dLower || !dDiag)
        return fail(CF_ERR_INVALID_ARG, "NULL argument");
    const size_t nb = sizeof(double) * c->n;
    const size_t fb = sizeof(double) * c->nf;
    CF_CUDA(cudaMemcpyAsync(c->d_io64, lambda, nb, cudaMemcpyHostToDevice, c->stream));
    CF_CUDA(cudaMemcpyAsync(c->d_io64b, x, nb, cudaMemcpyHostToDevice, c->stream));
    CF_TRY(launch_gradients(c, c->d_io64, c->d_io64b, c->d_gU, c->d_gL, c->d_gD));
    if (c->nf > 0)
    {
        CF_CUDA(cudaMemcpyAsync(dUpper, c->d_gU, fb, cudaMemcpyDeviceToHost, c->stream));
        CF_CUDA(cudaMemcpyAsync(dLower, c->d_gL, fb, cudaMemcpyDeviceToHost, c->stream));
    }
    CF_CUDA(cudaMemcpyAsync(dDiag, c->d_gD, nb, cudaMemcpyDeviceToHost, c->stream));
    CF_CUDA(cudaStreamSynchronize(c->stream));
    return CF_OK;
}

extern "C" int cf_solve_adjoint_device(cf_context* c, int32_t solver, const double* x,
                                       const double* dLdx, double* lambda, double* dUpper,
                                       double* dLower, double* dDiag, const cf_options* opts,
                                       cf_performance* perf)
{
    CF_TRY(check_ctx(c));
    if (!x || !dLdx || !lambda || !dUpper || !dLower || !dDiag || !opts || !perf)
        return fail(CF_ERR_INVALID_ARG, "NULL argument");
    CF_TRY(adjoint_solve(c, solver, dLdx, c->d_io64b, lambda, opts, perf));
    return launch_gradients(c, lambda, x, dUpper, dLower, dDiag);
}

extern "C" int cf_solve_adjoint(cf_context* c, int32_t solver, const double* x,
                                const double* dLdx, double* lambda, double* dUpper,
                                double* dLower, double* dDiag, const cf_options* opts,
                                cf_performance* perf)
{
    CF_TRY(check_ctx(c));
    if (!x || !dLdx || !lambda || !dUpper || !dLower || !dDiag || !opts || !perf)
        return fail(CF_ERR_INVALID_ARG, "NULL argument");
    const size_t nb = sizeof(double) * c->n;
    const size_t fb = sizeof(double) * c->nf;
    // dL/dx -> d_io64b, shifted source -> d_gD, lambda -> d_io64; then x ->
    // d_io64b and dDiag -> d_gD once those are free
    CF_CUDA(cudaMemcpyAsync(c->d_io64b, dLdx, nb, cudaMemcpyHostToDevice, c->stream));
    CF_TRY(adjoint_solve(c, solver, c->d_io64b, c->d_gD, c->d_io64, opts, perf));
    CF_CUDA(cudaMemcpyAsync(c->d_io64b, x, nb, cudaMemcpyHostToDevice, c->stream));
    CF_TRY(launch_gradients(c, c->d_io64, c->d_io64b, c->d_gU, c->d_gL, c->d_gD));
    CF_CUDA(cudaMemcpyAsync(lambda, c->d_io64, nb, cudaMemcpyDeviceToHost, c->stream));
    if (c->nf > 0)
    {
        CF_CUDA(cudaMemcpyAsync(dUpper, c->d_gU, fb, cudaMemcpyDeviceToHost, c->stream));
        CF_CUDA(cudaMemcpyAsync(dLower, c->d_gL, fb, cudaMemcpyDeviceToHost, c->stream));
    }
    CF_CUDA(cudaMemcpyAsync(dDiag, c->d_gD, nb, cudaMemcpyDeviceToHost, c->stream));
    CF_CUDA(cudaStreamSynchronize(c->stream));
    return CF_OK;
}
