// cf_persist.cu -- the inner PCG loop of a small mesh as ONE cooperative
// kernel.
//
// For meshes whose rows fit one per thread in a co-resident grid, the
// phases of an iteration (Chebyshev steps, p-update SpMV, update) run
// inside one launch separated by grid barriers,
// and the launch loops until the device-side stopping tests end the inner
// solve -- no kernel launch and no graph node per phase.  Each phase is the
// arithmetic of the corresponding kernel of cf_kernels.cuh on the same
// grid (one row per thread, ceil(n / 256) blocks), and the reductions are
// the same last-block folds, so a persistent inner solve returns exactly
// what the graph-driven one returns.
//
// Inside one launch, L1 is not coherent across SMs: every load of data that
// another block writes during the launch (vectors, partials, solver state)
// bypasses L1 (ld.global.cg, volatile state); data constant during the
// launch (matrix, diagonals, Chebyshev constants) keeps the read-only path.
//
// Grid barrier: generation counter in global memory; the last block to
// arrive resets the count and bumps the generation.  Every wait is bounded
// (the context's wait limit, default 2^24 polls with a short sleep each,
// cf_context_set_wait_limit); a block that gives up sets the error word and
// leaves, the others leave at their next barrier, and the host reports
// CF_ERR_DEVICE_TIMEOUT.  The launch is cooperative, so all blocks are
// co-resident and the default bound is never reached in normal runs.
//
// Opt-in (cf_options.persistentMaxCells > 0, cudaPCG): measured on B200 it
// is 20-35% slower than the graph-driven loop on 16k-64k-cell meshes (PCG,
// and BiCGStab before that loop was dropped from this file), whether the
// loads bypass L1 or not and whatever the barrier's
// polling interval -- a device-side graph launches the next kernel node
// faster than a grid barrier completes.
#include "cudafoam.h"
#include "cf_host.hpp"

#include <algorithm>
#include <string>

using namespace cf;

namespace {

constexpr int MW = MAXW_UNROLL;

using Bar = GridBar;   // cf_kernels.cuh

__device__ __forceinline__ float ld(const float* p) { return __ldcg(p); }

// ---------------------------------------------------------------- PCG

template <bool LAST>
__device__ __forceinline__ void p_cheb_step(const DevSell& A, const PcgBufs& B, const float* zin,
                                            const float* win, float* wout, float* zout, int j,
                                            volatile InnerState* st, unsigned int* ticket,
                                            double* part)
{
    const float c2 = __ldg(B.chebC + 2 * j - 1);
    const float c3 = __ldg(B.chebC + 2 * j);
    double acc[1] = {0.0};
    CF_ROWS(row, A.n)
    {
        const float zr = ld(zin + row);
        const float v = row_f32<MW>(A, row, __fmul_rn(__ldg(B.diag + row), zr),
                                    [&](int c) { return ld(zin + c); });
        const float r = ld(B.rA + row);
        const float wn = __fadd_rn(__fmul_rn(c2, ld(win + row)),
                                   __fmul_rn(__fmul_rn(c3, __ldg(B.rD + row)), __fsub_rn(r, v)));
        const float zn = __fadd_rn(zr, wn);
        wout[row] = wn;
        zout[row] = zn;
        if (LAST) acc[0] += (double)zn * (double)r;
    }
    if (LAST)
    {
        if (grid_sum<1>(acc, part, ticket) && threadIdx.x == 0)
        {
            st->wArAold = st->wArA;
            st->wArA = acc[0];
            st->beta = (st->it == 0) ? 0.0 : st->wArA / st->wArAold;
        }
    }
}

__device__ __forceinline__ void p_pcg_p_spmv(const DevSell& A, const PcgBufs& B, const float* wA,
                                             volatile InnerState* st, unsigned int* ticket,
                                             double* part)
{
    const int n = A.n;
    const int par = st->it & 1;
    const float* Pold = B.P + (size_t)(par ^ 1) * n;
    float* Pn = B.P + (size_t)par * n;
    const float beta = (float)st->beta;
    auto pf = [&](int c) { return __fadd_rn(ld(wA + c), __fmul_rn(beta, ld(Pold + c))); };
    double acc[1] = {0.0};
    CF_ROWS(row, n)
    {
        const float pr = pf(row);
        const float y = row_f32<MW>(A, row, __fmul_rn(__ldg(B.diag + row), pr), pf);
        Pn[row] = pr;
        B.Q[row] = y;
        acc[0] += (double)pr * (double)y;
    }
    if (grid_sum<1>(acc, part, ticket) && threadIdx.x == 0)
    {
        st->wApA = acc[0];
        st->alpha = st->wArA / st->wApA;
    }
}

template <bool CHEB>
__device__ __forceinline__ void p_pcg_update(const PcgBufs& B, volatile InnerState* st,
                                             unsigned int* ticket, double* part)
{
    const int n = B.n;
    const int par = st->it & 1;
    const float* P = B.P + (size_t)par * n;
    const float* D = B.D + (size_t)st->cur * n;
    float* Dn = B.D + (size_t)st->nxt * n;
    const float alpha = (float)st->alpha;
    const float c1 = CHEB ? __ldg(B.chebC) : 0.0f;
    double acc[2] = {0.0, 0.0};
    CF_ROWS(row, n)
    {
        Dn[row] = __fadd_rn(ld(D + row), __fmul_rn(alpha, ld(P + row)));
        const float rn = __fsub_rn(ld(B.rA + row), __fmul_rn(alpha, ld(B.Q + row)));
        B.rA[row] = rn;
        acc[0] += (double)fabsf(rn);
        if (CHEB)
        {
            B.W0[row] = __fmul_rn(__fmul_rn(c1, __ldg(B.rD + row)), rn);
        }
        else
        {
            const float wa = __fmul_rn(rn, __ldg(B.rD + row));
            B.W0[row] = wa;
            acc[1] += (double)wa * (double)rn;
        }
    }
    if (grid_sum<2>(acc, part, ticket) && threadIdx.x == 0)
    {
        st->res = acc[0];
        if (!CHEB)
        {
            st->wArAold = st->wArA;
            st->wArA = acc[1];
            st->beta = st->wArA / st->wArAold;
        }
        st->cur = st->nxt;
        st->it = st->it + 1;
        inner_sync_point(st, true);
    }
}

// launch_pcg_body's phases, repeated until the inner solve is done
template <bool CHEB>
__global__ void __launch_bounds__(NT) kp_pcg(DevSell A, PcgBufs B, int order, InnerState* stp,
                                             double* part, Bar bar)
{
    volatile InnerState* st = stp;
    unsigned int* ticket = &stp->ticket;
    float* Z[2] = {B.Z0, B.Z1};
    while (!st->done)
    {
        if (CHEB)
        {
            for (int j = 1; j < order; ++j)
            {
                const float* zin = (j == 1) ? B.W0 : Z[(j - 1) & 1];
                const float* win = (j == 1) ? B.W0 : B.W1;
                if (j == order - 1)
                    p_cheb_step<true>(A, B, zin, win, B.W1, Z[j & 1], j, st, ticket, part);
                else
                    p_cheb_step<false>(A, B, zin, win, B.W1, Z[j & 1], j, st, ticket, part);
                if (!grid_barrier(bar)) return;
            }
        }
        p_pcg_p_spmv(A, B, CHEB ? Z[(order - 1) & 1] : B.W0, st, ticket, part);
        if (!grid_barrier(bar)) return;
        p_pcg_update<CHEB>(B, st, ticket, part);
        if (!grid_barrier(bar)) return;
    }
}

}  // namespace

namespace cf {

int persistent_inner(cf_context* c, int kind, int order, int maxCells, bool* ran)
{
    *ran = false;
    if (kind != 0 || maxCells <= 0 || c->n > maxCells || !c->coopLaunch || !c->d_bar)
        return CF_OK;
    const int n = c->n;
    const int need = (n + NT - 1) / NT;
    // the phase kernels of the graph path run on `need` blocks exactly
    // when each one's resident capacity covers it; the persistent grid must
    // be co-resident
    const void* fn = order > 1 ? (const void*)kp_pcg<true> : (const void*)kp_pcg<false>;
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, NT, 0) != cudaSuccess)
    {
        cudaGetLastError();
        return CF_OK;
    }
    if ((long long)occ * c->numSMs < need) return CF_OK;
    const void* phases[4] = {(const void*)k_cheb_step<true, MW>, (const void*)k_cheb_step<false, MW>,
                             (const void*)k_pcg_p_spmv<MW>,
                             order > 1 ? (const void*)k_pcg_update<true>
                                       : (const void*)k_pcg_update<false>};
    const int np = 4;
    for (int i = 0; i < np; ++i)
        if (grid_for(c, phases[i], n) != need) return CF_OK;

    cudaStream_t s = c->stream;
    if (cudaMemsetAsync(c->d_bar, 0, sizeof(unsigned int) * 4, s) != cudaSuccess)
        return fail(CF_ERR_CUDA, "cudaMemsetAsync (grid barrier)");
    const DevSell A = sell_of(c);
    Bar bar{c->d_bar, c->d_bar + 1, reinterpret_cast<int*>(c->d_bar + 2),
            (unsigned long long)c->waitPolls};
    PcgBufs B = pcg_bufs(c);
    InnerState* st = c->d_st;
    double* part = c->d_part;
    int ord = order;
    void* args[] = {(void*)&A, (void*)&B, (void*)&ord, (void*)&st, (void*)&part, (void*)&bar};
    const cudaError_t e = cudaLaunchCooperativeKernel(fn, dim3(need), dim3(NT), args, 0, s);
    if (e != cudaSuccess)
        return fail(CF_ERR_CUDA, std::string("cudaLaunchCooperativeKernel: ") + cudaGetErrorString(e));
    c->launches++;
    *ran = true;
    return CF_OK;
}

int persistent_status(cf_context* c)
{
    int err = 0;
    if (cudaMemcpy(&err, c->d_bar + 2, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
        return fail(CF_ERR_CUDA, "reading the grid-barrier status");
    if (err) return fail(CF_ERR_DEVICE_TIMEOUT, "a grid barrier of the persistent inner solve timed out");
    return CF_OK;
}

}  // namespace cf
