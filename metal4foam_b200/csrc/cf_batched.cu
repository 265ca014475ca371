// cf_batched.cu -- many independent pressure systems solved together.
//
// No counterpart in the reference (the design's batching row): the
// reference solves one system per call with one host sync per iteration.
// Here a batch of independent meshes of any sizes runs through one set of
// kernels: each phase of the Krylov iteration is ONE launch over every row
// of every still-active system, the iterations run in a CUDA-graph WHILE
// loop until the last system has finished, and every per-system decision of
// the FP64 driver (deflation, Gershgorin bound, restarts, constant-mode
// shift, polish, convergence) is a per-system state machine on the device.
//
// Layout: the systems' SELL-32 layouts are concatenated; system s owns the
// global rows [row0, row0 + npad) with npad = n rounded up to whole slices,
// so no slice and no 256-row tile spans two systems.  A tile = (system,
// first row); reductions are per system: each tile writes one FP64 partial,
// the last tile of a system to finish (per-system atomic ticket) folds the
// system's partials in tile order and updates that system's scalars.
// Per row the arithmetic is the single-system kernels' (same row functions),
// so every system follows exactly the iteration it would follow alone.
#include "cudafoam.h"
#include "cf_host.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <thread>
#include <vector>

using namespace cf;

namespace {

constexpr int MW = MAXW_UNROLL;
// default solo threshold: this many NT-row blocks per SM
constexpr int SOLO_BLOCKS_PER_SM = 3;

struct BSys
{
    int row0, n, npad, tile0, ntiles, face0, nf;
};

// per-system FP64 driver state (metalFoamSolver.C:101-415, one per system)
struct BDrv
{
    double xbar, normFactor, initRes, finalRes, prevRes, rmean, dmean, ur, uu, l2r, l2b;
    double chebBeta, target, finalResSum32;
    long long nPinned;
    int signflip, deflate, polished, solved, finished, singular, stagnated, totalIter;
    int nRestarts, restage, ranInner;
    unsigned int ticket;
};

struct BArgs
{
    int nTiles;
    const int2* tiles;
    const BSys* sys;
    DevSell A;
    long long N;            // global rows (buffer stride)
    const float* diag32;
    const float* rD;
    const float* chebC;     // [S][2 * CF_MAX_CHEB]
    float* rA;
    float* W0;
    float* W1;
    float* Z0;
    float* Z1;
    float* P;               // [2N]
    float* Q;
    float* D;               // [3N]
    double* r64;
    double* psi;
    double* b;
    double* u;
    double* diag64;
    InnerState* st;
    BDrv* drv;
    double* part;           // [NPART][nTiles]
    int* counters;          // [0] inner-active systems, [1] unfinished systems,
                            // [2] active tiles, [3] active-tile list stale
    int* actTiles;          // [nTiles] tiles of inner-active systems (first [2])
};

constexpr int kChebStride = 2 * CF_MAX_CHEB;
// rows per tile: 8 per thread; one per-system partial per tile
constexpr int kTileRows = 8 * NT;

// Per-system sum of NR values over the tiles of one kernel launch.  Returns
// true in the block that processed the system's last tile; its thread 0
// then holds the totals.
template <int NR>
__device__ __forceinline__ bool sys_sum(double (&v)[NR], const BArgs& B, int t, int s,
                                        unsigned int* ticket)
{
    __shared__ bool amLast;
    block_sum<NR>(v);
    const BSys sy = B.sys[s];
    if (threadIdx.x == 0)
    {
#pragma unroll
        for (int r = 0; r < NR; ++r) B.part[(size_t)r * B.nTiles + t] = v[r];
        __threadfence();
        const unsigned int k = atomicAdd(ticket, 1u);
        amLast = (k == (unsigned)sy.ntiles - 1);
    }
    __syncthreads();
    if (!amLast) return false;
    __threadfence();
    double acc[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) acc[r] = 0.0;
    for (int i = threadIdx.x; i < sy.ntiles; i += NT)
    {
#pragma unroll
        for (int r = 0; r < NR; ++r) acc[r] += __ldcg(B.part + (size_t)r * B.nTiles + sy.tile0 + i);
    }
    block_sum<NR>(acc);
    if (threadIdx.x == 0)
    {
#pragma unroll
        for (int r = 0; r < NR; ++r) v[r] = acc[r];
        *ticket = 0u;
    }
    return true;
}

__device__ __forceinline__ double sys_max(double v, const BArgs& B, int t, int s,
                                          unsigned int* ticket, bool* last)
{
    __shared__ double sh[NT / 32];
    __shared__ bool amLast;
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    const BSys sy = B.sys[s];
    __syncthreads();
    v = warp_max(v);
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    if (threadIdx.x == 0)
    {
        double m = sh[0];
        for (int w = 1; w < NT / 32; ++w) m = fmax(m, sh[w]);
        B.part[t] = m;
        __threadfence();
        amLast = atomicAdd(ticket, 1u) == (unsigned)sy.ntiles - 1;
    }
    __syncthreads();
    *last = amLast;
    if (!amLast) return 0.0;
    __threadfence();
    double m = -INFINITY;
    for (int i = threadIdx.x; i < sy.ntiles; i += NT) m = fmax(m, __ldcg(B.part + sy.tile0 + i));
    m = warp_max(m);
    __syncthreads();
    if (lane == 0) sh[wid] = m;
    __syncthreads();
    double res = 0.0;
    if (threadIdx.x == 0)
    {
        res = sh[0];
        for (int w = 1; w < NT / 32; ++w) res = fmax(res, sh[w]);
        *ticket = 0u;
    }
    return res;
}

#define CFB_TILE_BEGIN(t)                                             \
    for (int t = blockIdx.x; t < B.nTiles; t += gridDim.x)            \
    {                                                                 \
        const int s = B.tiles[t].x;                                   \
        const int tileRow = B.tiles[t].y;                             \
        const BSys sy = B.sys[s];                                     \
        const int tileEnd = min(tileRow + kTileRows, sy.row0 + sy.n);

// the same over the compacted list of tiles of inner-active systems
#define CFB_ACTIVE_BEGIN(t)                                           \
    const int nAct_ = B.counters[2];                                  \
    for (int k_ = blockIdx.x; k_ < nAct_; k_ += gridDim.x)            \
    {                                                                 \
        const int t = B.actTiles[k_];                                 \
        const int s = B.tiles[t].x;                                   \
        const int tileRow = B.tiles[t].y;                             \
        const BSys sy = B.sys[s];                                     \
        const int tileEnd = min(tileRow + kTileRows, sy.row0 + sy.n);

// the real rows of the current tile owned by this thread
#define CFB_ROWS for (int row = tileRow + (int)threadIdx.x; row < tileEnd; row += NT)

#define CFB_TILE_END }

// ------------------------------------------------------------ staging / driver

__global__ void kb_gather(long long N, const int* __restrict__ perm, const double* __restrict__ src,
                          double* __restrict__ dst)
{
    for (long long r = (long long)blockIdx.x * NT + threadIdx.x; r < N; r += (long long)gridDim.x * NT)
    {
        const int p = perm[r];
        dst[r] = p >= 0 ? src[p] : 0.0;
    }
}

__global__ void kb_scatter(long long N, const int* __restrict__ perm, const double* __restrict__ src,
                           double* __restrict__ dst)
{
    for (long long r = (long long)blockIdx.x * NT + threadIdx.x; r < N; r += (long long)gridDim.x * NT)
    {
        const int p = perm[r];
        if (p >= 0) dst[p] = src[r];
    }
}

template <int MAXW>
__global__ void __launch_bounds__(NT) kb_sumA(BArgs B)
{
    CFB_TILE_BEGIN(t)
    double acc[2] = {0.0, 0.0};
    CFB_ROWS
    {
        const double d = B.diag64[row];
        const double sm = row_f64<MAXW>(B.A, B.A.val64, row, d, [](int) { return 1.0; });
        B.u[row] = sm;
        if (fabs(sm) > 1e-8 * fabs(d)) acc[0] += 1.0;
        const double d0 = __dsub_rn(d, sm);
        if (__dmul_rn(d0, d) <= VSMALL * fabs(d0)) acc[1] += 1.0;
    }
    if (sys_sum<2>(acc, B, t, s, &B.drv[s].ticket) && threadIdx.x == 0)
    {
        B.drv[s].nPinned = (long long)acc[0];
        B.drv[s].signflip = acc[1] > 0.0;
    }
    CFB_TILE_END
}

// per-system mean: WHICH 0 = psi (xbar, all systems), 1 = r64 (rmean,
// deflated unfinished systems)
template <int WHICH>
__global__ void __launch_bounds__(NT) kb_mean(BArgs B)
{
    CFB_TILE_BEGIN(t)
    if (WHICH == 1 && (B.drv[s].finished || !B.drv[s].deflate)) continue;
    double acc[1] = {0.0};
    CFB_ROWS acc[0] += WHICH == 0 ? B.psi[row] : B.r64[row];
    if (sys_sum<1>(acc, B, t, s, &B.drv[s].ticket) && threadIdx.x == 0)
    {
        const double m = acc[0] / (double)sy.n;
        if (WHICH == 0)
            B.drv[s].xbar = m;
        else
            B.drv[s].rmean = m;
    }
    CFB_TILE_END
}

template <int MAXW>
__global__ void __launch_bounds__(NT) kb_residual0(BArgs B)
{
    CFB_TILE_BEGIN(t)
    double acc[2] = {0.0, 0.0};
    CFB_ROWS
    {
        const double* psi = B.psi;
        const double wa = row_f64<MAXW>(B.A, B.A.val64, row, __dmul_rn(B.diag64[row], psi[row]),
                                        [&](int c) { return __ldg(psi + c); });
        const double bb = B.b[row];
        const double rr = __dsub_rn(bb, wa);
        B.r64[row] = rr;
        const double pA = __dmul_rn(B.u[row], B.drv[s].xbar);
        acc[0] += __dadd_rn(fabs(__dsub_rn(wa, pA)), fabs(__dsub_rn(bb, pA)));
        acc[1] += fabs(rr);
    }
    if (sys_sum<2>(acc, B, t, s, &B.drv[s].ticket) && threadIdx.x == 0)
    {
        BDrv& d = B.drv[s];
        d.normFactor = acc[0] + 1e-20;
        d.initRes = acc[1] / d.normFactor;
        d.finalRes = d.initRes;
    }
    CFB_TILE_END
}

__device__ __forceinline__ bool converged_(double tol, double relTol, double init, double fin)
{
    return (fin < tol) || (relTol > 1e-20 && fin < relTol * init);
}

// entry decisions per system (metalFoamSolver.C:131-257)
__global__ void kb_entry(int S, BDrv* drv, cf_options o)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S) return;
    BDrv& d = drv[s];
    d.solved = (o.minIter > 0) || !converged_(o.tolerance, o.relTol, d.initRes, d.finalRes);
    d.finished = !d.solved;
    d.totalIter = 0;
    d.nRestarts = 0;
    d.polished = 0;
    d.singular = 0;
    d.stagnated = 0;
    d.restage = 0;
    d.chebBeta = 2.0;
    d.finalResSum32 = 0.0;
    d.prevRes = d.initRes;
    d.target = fmax(o.tolerance, o.relTol * d.initRes) * d.normFactor;
    d.deflate = (o.deflate == CF_DEFLATE_ON) ? 1 : 0;   // auto: kb_entry_auto
}

__global__ void kb_entry_auto(int S, const BSys* sys, BDrv* drv, int deflateOpt)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S) return;
    BDrv& d = drv[s];
    if (deflateOpt == CF_DEFLATE_AUTO) d.deflate = (10LL * d.nPinned <= (long long)sys[s].n);
    if (d.deflate && d.signflip) d.deflate = 0;
}

// FP32 diagonal per system (restageOnly: systems flagged by the polish)
__global__ void kb_stage_diag32(BArgs B, float* diag32, float* rD, int restageOnly)
{
    CFB_TILE_BEGIN(t)
    if (restageOnly && !B.drv[s].restage) continue;
    CFB_ROWS
    {
        const double dp = B.drv[s].deflate ? __dsub_rn(B.diag64[row], B.u[row]) : B.diag64[row];
        diag32[row] = (float)dp;
        rD[row] = (float)(1.0 / dp);
    }
    CFB_TILE_END
}

template <int MAXW>
__global__ void __launch_bounds__(NT) kb_gershgorin(BArgs B, const int* __restrict__ eface,
                                                    const double* __restrict__ upper, int order,
                                                    double ratio, float* chebC)
{
    CFB_TILE_BEGIN(t)
    double m = 0.0;
    CFB_ROWS
    {
        const int sl = row >> 5;
        const int b0 = B.A.sliceOff[sl];
        const int w = (B.A.sliceOff[sl + 1] - b0) >> 5;
        const int base = b0 + (row & 31);
        double so = 0.0;
        for (int k = 0; k < w; ++k)
        {
            const int c = B.A.col[base + SLICE * k];
            if (is_nbr(c)) so = __dadd_rn(so, fabs(upper[eface[base + SLICE * k]]));
        }
        for (int k = 0; k < w; ++k)
        {
            const int c = B.A.col[base + SLICE * k];
            if (is_own(c)) so = __dadd_rn(so, fabs(upper[eface[base + SLICE * k]]));
        }
        const double dp = B.drv[s].deflate ? __dsub_rn(B.diag64[row], B.u[row]) : B.diag64[row];
        m = fmax(m, __dadd_rn(1.0, so / fabs(dp)));
    }
    bool last = false;
    const double mx = sys_max(m, B, t, s, &B.drv[s].ticket, &last);
    if (last && threadIdx.x == 0)
    {
        B.drv[s].chebBeta = mx;
        cheb_constants(order, mx, ratio, chebC + (size_t)s * kChebStride);
    }
    CFB_TILE_END
}

// start of an outer pass: inner setup per unfinished system
__global__ void kb_outer_begin(int S, InnerState* st, BDrv* drv, int* counters, int maxIter,
                               int ips, int stagLimit)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S) return;
    BDrv& d = drv[s];
    InnerState& q = st[s];
    q.wArA = q.wArAold = q.wApA = q.alpha = q.beta = q.res = 0.0;
    q.bestRes = 1.0e300;
    q.finalResSum = 0.0;
    q.it = 0;
    q.ips = ips < 1 ? 1 : ips;
    q.stagLimit = stagLimit > 0 ? stagLimit : STAG_LIMIT;
    q.lastSync = 0;
    q.noProgress = 0;
    q.cur = 0;
    q.best = 0;
    q.nxt = 1;
    q.converged = q.singular = q.stagnated = q.early = 0;
    q.sel = 0;
    q.ticket = 0u;
    q.target = d.target;
    q.maxIter = maxIter - d.totalIter;
    d.restage = 0;
    d.ranInner = !d.finished;
    if (d.finished || q.maxIter <= 0)
    {
        q.done = 1;
    }
    else
    {
        q.done = 0;
        atomicAdd(&counters[0], 1);
    }
}

template <bool CHEB>
__global__ void __launch_bounds__(NT) kb_pcg_init(BArgs B)
{
    CFB_TILE_BEGIN(t)
    if (!B.drv[s].ranInner) continue;
    const float c1 = CHEB ? B.chebC[(size_t)s * kChebStride] : 0.0f;
    const double m = B.drv[s].deflate ? B.drv[s].rmean : 0.0;
    double acc[1] = {0.0};
    CFB_ROWS
    {
        const float ra = (float)(B.r64[row] - m);
        B.rA[row] = ra;
        B.D[row] = 0.0f;
        B.P[row] = 0.0f;
        B.P[B.N + row] = 0.0f;
        if (CHEB)
        {
            B.W0[row] = __fmul_rn(__fmul_rn(c1, B.rD[row]), ra);
        }
        else
        {
            const float wa = __fmul_rn(ra, B.rD[row]);
            B.W0[row] = wa;
            acc[0] += (double)wa * (double)ra;
        }
    }
    if (!CHEB)
    {
        if (sys_sum<1>(acc, B, t, s, &B.st[s].ticket) && threadIdx.x == 0)
        {
            B.st[s].wArAold = B.st[s].wArA;
            B.st[s].wArA = acc[0];
            B.st[s].beta = 0.0;
        }
    }
    CFB_TILE_END
}

template <bool LAST, int MAXW>
__global__ void __launch_bounds__(NT) kb_cheb_step(BArgs B, const float* zin, const float* win,
                                                   float* wout, float* zout, int j)
{
    CFB_ACTIVE_BEGIN(t)
    if (B.st[s].done) continue;
    const float* cc = B.chebC + (size_t)s * kChebStride;
    const float c2 = cc[2 * j - 1];
    const float c3 = cc[2 * j];
    double acc[1] = {0.0};
    CFB_ROWS
    {
        const float zr = zin[row];
        const float v = row_f32<MAXW>(B.A, row, __fmul_rn(B.diag32[row], zr),
                                      [&](int c) { return __ldg(zin + c); });
        const float r = B.rA[row];
        const float wn = __fadd_rn(__fmul_rn(c2, win[row]),
                                   __fmul_rn(__fmul_rn(c3, B.rD[row]), __fsub_rn(r, v)));
        const float zn = __fadd_rn(zr, wn);
        wout[row] = wn;
        zout[row] = zn;
        if (LAST) acc[0] += (double)zn * (double)r;
    }
    if (LAST)
    {
        if (sys_sum<1>(acc, B, t, s, &B.st[s].ticket) && threadIdx.x == 0)
        {
            InnerState& q = B.st[s];
            q.wArAold = q.wArA;
            q.wArA = acc[0];
            q.beta = (q.it == 0) ? 0.0 : q.wArA / q.wArAold;
        }
    }
    CFB_TILE_END
}

// The Chebyshev steps without the z.r sum, one row per thread per pass (as
// the single-system kernels): sub-tile q (NT rows) is the rows
// NT (q mod SUB) .. + NT of active tile q / SUB; block b takes the
// sub-tiles b, b + gridDim.x, ...  Same arithmetic per row as kb_cheb_step.
constexpr int kSubTiles = kTileRows / NT;

template <int MAXW>
__global__ void __launch_bounds__(NT) kb_cheb_step_rows(BArgs B, const float* zin, const float* win,
                                                        float* wout, float* zout, int j)
{
    const int nSub = B.counters[2] * kSubTiles;
    for (int q = blockIdx.x; q < nSub; q += gridDim.x)
    {
        const int t = B.actTiles[q / kSubTiles];
        const int s = B.tiles[t].x;
        if (B.st[s].done) continue;
        const BSys sy = B.sys[s];
        const int row = B.tiles[t].y + (q % kSubTiles) * NT + (int)threadIdx.x;
        if (row >= sy.row0 + sy.n) continue;
        const float* cc = B.chebC + (size_t)s * kChebStride;
        const float c2 = cc[2 * j - 1];
        const float c3 = cc[2 * j];
        const float zr = zin[row];
        const float v = row_f32<MAXW>(B.A, row, __fmul_rn(B.diag32[row], zr),
                                      [&](int c) { return __ldg(zin + c); });
        const float r = B.rA[row];
        const float wn = __fadd_rn(__fmul_rn(c2, win[row]),
                                   __fmul_rn(__fmul_rn(c3, B.rD[row]), __fsub_rn(r, v)));
        wout[row] = wn;
        zout[row] = __fadd_rn(zr, wn);
    }
}

template <int MAXW>
__global__ void __launch_bounds__(NT) kb_pcg_p_spmv(BArgs B, const float* wA)
{
    CFB_ACTIVE_BEGIN(t)
    if (B.st[s].done) continue;
    const int par = B.st[s].it & 1;
    const float* __restrict__ Pold = B.P + (size_t)(par ^ 1) * B.N;
    float* __restrict__ Pn = B.P + (size_t)par * B.N;
    const float beta = (float)B.st[s].beta;
    double acc[1] = {0.0};
    CFB_ROWS
    {
        auto pf = [&](int c) { return __fadd_rn(__ldg(wA + c), __fmul_rn(beta, __ldg(Pold + c))); };
        const float pr = pf(row);
        const float y = row_f32<MAXW>(B.A, row, __fmul_rn(B.diag32[row], pr), pf);
        Pn[row] = pr;
        B.Q[row] = y;
        acc[0] += (double)pr * (double)y;
    }
    if (sys_sum<1>(acc, B, t, s, &B.st[s].ticket) && threadIdx.x == 0)
    {
        InnerState& q = B.st[s];
        q.wApA = acc[0];
        q.alpha = q.wArA / q.wApA;
    }
    CFB_TILE_END
}

template <bool CHEB>
__global__ void __launch_bounds__(NT) kb_pcg_update(BArgs B, cudaGraphConditionalHandle h,
                                                    int useCond)
{
    CFB_ACTIVE_BEGIN(t)
    if (B.st[s].done) continue;
    InnerState& q = B.st[s];
    const int par = q.it & 1;
    const float* __restrict__ Pv = B.P + (size_t)par * B.N;
    const float* __restrict__ Dc = B.D + (size_t)q.cur * B.N;
    float* __restrict__ Dn = B.D + (size_t)q.nxt * B.N;
    const float alpha = (float)q.alpha;
    const float c1 = CHEB ? B.chebC[(size_t)s * kChebStride] : 0.0f;
    double acc[2] = {0.0, 0.0};
    CFB_ROWS
    {
        Dn[row] = __fadd_rn(Dc[row], __fmul_rn(alpha, Pv[row]));
        const float rn = __fsub_rn(B.rA[row], __fmul_rn(alpha, B.Q[row]));
        B.rA[row] = rn;
        acc[0] += (double)fabsf(rn);
        if (CHEB)
        {
            B.W0[row] = __fmul_rn(__fmul_rn(c1, B.rD[row]), rn);
        }
        else
        {
            const float wa = __fmul_rn(rn, B.rD[row]);
            B.W0[row] = wa;
            acc[1] += (double)wa * (double)rn;
        }
    }
    if (sys_sum<2>(acc, B, t, s, &q.ticket) && threadIdx.x == 0)
    {
        q.res = acc[0];
        if (!CHEB)
        {
            q.wArAold = q.wArA;
            q.wArA = acc[1];
            q.beta = q.wArA / q.wArAold;
        }
        q.cur = q.nxt;
        q.it = q.it + 1;
        inner_sync_point(&q, true);
        if (q.done)
        {
            B.counters[3] = 1;   // the active-tile list needs rebuilding
            const int left = atomicSub(&B.counters[0], 1) - 1;
            if (left == 0 && useCond) cudaGraphSetConditional(h, 0u);
        }
    }
    CFB_TILE_END
}

// Rebuild the list of tiles whose system is still iterating (one block;
// runs after every update, returns at once unless a system finished or
// `force`).  List order does not matter: partial sums are stored by tile id
// and folded in tile order.
__global__ void __launch_bounds__(1024) kb_compact(BArgs B, int force)
{
    __shared__ int count;
    if (!force && B.counters[3] == 0) return;
    if (threadIdx.x == 0) count = 0;
    __syncthreads();
    for (int t = threadIdx.x; t < B.nTiles; t += blockDim.x)
    {
        const int s = B.tiles[t].x;
        if (!B.st[s].done) B.actTiles[atomicAdd(&count, 1)] = t;
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        B.counters[2] = count;
        B.counters[3] = 0;
    }
}

// ------------------------------------------------ one persistent launch
//
// The inner loop of every system of the batch as ONE cooperative kernel:
// the phases of an iteration (Chebyshev steps, p-update SpMV, update) over
// the active tiles, separated by bounded grid barriers, then block 0
// rebuilds the active-tile list -- what the graph loop's kernels do, in the
// same per-row arithmetic and the same per-tile partial sums folded in tile
// order, so every system gets bit for bit what the graph loop gives it.
// Inside one launch L1 is not coherent across SMs: every load of data that
// another block writes during the launch (vectors, partials, states, the
// tile list) bypasses L1 (ld.global.cg, volatile); the matrix, diagonals,
// constants and the tile table keep the read-only path.

__device__ __forceinline__ float ldv(const float* p) { return __ldcg(p); }

#define CFBP_ACTIVE_BEGIN(t)                                          \
    const int nAct_ = *(volatile int*)&B.counters[2];                 \
    for (int k_ = blockIdx.x; k_ < nAct_; k_ += gridDim.x)            \
    {                                                                 \
        const int t = __ldcg(B.actTiles + k_);                        \
        const int s = __ldg(&B.tiles[t].x);                           \
        const int tileRow = __ldg(&B.tiles[t].y);                     \
        const BSys sy = B.sys[s];                                     \
        const int tileEnd = min(tileRow + kTileRows, sy.row0 + sy.n); \
        volatile InnerState* vq = B.st + s;

template <bool LAST, int MAXW>
__device__ __forceinline__ void kbp_cheb_step(const BArgs& B, const float* zin, const float* win,
                                              float* wout, float* zout, int j)
{
    CFBP_ACTIVE_BEGIN(t)
    if (vq->done) continue;
    const float* cc = B.chebC + (size_t)s * kChebStride;
    const float c2 = __ldg(cc + 2 * j - 1);
    const float c3 = __ldg(cc + 2 * j);
    double acc[1] = {0.0};
    CFB_ROWS
    {
        const float zr = ldv(zin + row);
        const float v = row_f32<MAXW>(B.A, row, __fmul_rn(__ldg(B.diag32 + row), zr),
                                      [&](int c) { return ldv(zin + c); });
        const float r = ldv(B.rA + row);
        const float wn = __fadd_rn(__fmul_rn(c2, ldv(win + row)),
                                   __fmul_rn(__fmul_rn(c3, __ldg(B.rD + row)), __fsub_rn(r, v)));
        const float zn = __fadd_rn(zr, wn);
        wout[row] = wn;
        zout[row] = zn;
        if (LAST) acc[0] += (double)zn * (double)r;
    }
    if (LAST)
    {
        if (sys_sum<1>(acc, B, t, s, &B.st[s].ticket) && threadIdx.x == 0)
        {
            vq->wArAold = vq->wArA;
            vq->wArA = acc[0];
            vq->beta = (vq->it == 0) ? 0.0 : vq->wArA / vq->wArAold;
        }
    }
    CFB_TILE_END
}

template <int MAXW>
__device__ __forceinline__ void kbp_pcg_p_spmv(const BArgs& B, const float* wA)
{
    CFBP_ACTIVE_BEGIN(t)
    if (vq->done) continue;
    const int par = vq->it & 1;
    const float* Pold = B.P + (size_t)(par ^ 1) * B.N;
    float* Pn = B.P + (size_t)par * B.N;
    const float beta = (float)vq->beta;
    double acc[1] = {0.0};
    CFB_ROWS
    {
        auto pf = [&](int c) { return __fadd_rn(ldv(wA + c), __fmul_rn(beta, ldv(Pold + c))); };
        const float pr = pf(row);
        const float y = row_f32<MAXW>(B.A, row, __fmul_rn(__ldg(B.diag32 + row), pr), pf);
        Pn[row] = pr;
        B.Q[row] = y;
        acc[0] += (double)pr * (double)y;
    }
    if (sys_sum<1>(acc, B, t, s, &B.st[s].ticket) && threadIdx.x == 0)
    {
        vq->wApA = acc[0];
        vq->alpha = vq->wArA / vq->wApA;
    }
    CFB_TILE_END
}

template <bool CHEB>
__device__ __forceinline__ void kbp_pcg_update(const BArgs& B)
{
    CFBP_ACTIVE_BEGIN(t)
    if (vq->done) continue;
    const int par = vq->it & 1;
    const float* Pv = B.P + (size_t)par * B.N;
    const float* Dc = B.D + (size_t)vq->cur * B.N;
    float* Dn = B.D + (size_t)vq->nxt * B.N;
    const float alpha = (float)vq->alpha;
    const float c1 = CHEB ? __ldg(B.chebC + (size_t)s * kChebStride) : 0.0f;
    double acc[2] = {0.0, 0.0};
    CFB_ROWS
    {
        Dn[row] = __fadd_rn(ldv(Dc + row), __fmul_rn(alpha, ldv(Pv + row)));
        const float rn = __fsub_rn(ldv(B.rA + row), __fmul_rn(alpha, ldv(B.Q + row)));
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
    if (sys_sum<2>(acc, B, t, s, &B.st[s].ticket) && threadIdx.x == 0)
    {
        vq->res = acc[0];
        if (!CHEB)
        {
            vq->wArAold = vq->wArA;
            vq->wArA = acc[1];
            vq->beta = vq->wArA / vq->wArAold;
        }
        vq->cur = vq->nxt;
        vq->it = vq->it + 1;
        inner_sync_point(vq, true);
        if (vq->done)
        {
            *(volatile int*)&B.counters[3] = 1;
            atomicSub(&B.counters[0], 1);
        }
    }
    CFB_TILE_END
}

// kb_compact inside the persistent launch (block 0, NT threads)
__device__ __forceinline__ void kbp_compact(const BArgs& B)
{
    __shared__ int count;
    if (*(volatile int*)&B.counters[3] == 0) return;
    if (threadIdx.x == 0) count = 0;
    __syncthreads();
    for (int t = threadIdx.x; t < B.nTiles; t += NT)
    {
        const int s = __ldg(&B.tiles[t].x);
        if (!((volatile InnerState*)(B.st + s))->done) B.actTiles[atomicAdd(&count, 1)] = t;
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        *(volatile int*)&B.counters[2] = count;
        *(volatile int*)&B.counters[3] = 0;
    }
    __syncthreads();
}

template <bool CHEB, int MAXW>
__global__ void __launch_bounds__(NT) kbp_pcg(BArgs B, int order, GridBar bar)
{
    float* Z[2] = {B.Z0, B.Z1};
    // counters[0] (systems still iterating) changes only in the update
    // phase; every block reads it after the same barrier
    while (*(volatile int*)&B.counters[0] > 0)
    {
        const float* wA = B.W0;
        if (CHEB)
        {
            for (int j = 1; j < order; ++j)
            {
                const float* zin = (j == 1) ? B.W0 : Z[(j - 1) & 1];
                const float* win = (j == 1) ? B.W0 : B.W1;
                if (j == order - 1)
                    kbp_cheb_step<true, MAXW>(B, zin, win, B.W1, Z[j & 1], j);
                else
                    kbp_cheb_step<false, MAXW>(B, zin, win, B.W1, Z[j & 1], j);
                if (!grid_barrier(bar)) return;
            }
            wA = Z[(order - 1) & 1];
        }
        kbp_pcg_p_spmv<MAXW>(B, wA);
        if (!grid_barrier(bar)) return;
        kbp_pcg_update<CHEB>(B);
        if (!grid_barrier(bar)) return;
        if (blockIdx.x == 0) kbp_compact(B);
        if (!grid_barrier(bar)) return;
    }
}

__global__ void kb_inner_final(int S, InnerState* st, BDrv* drv)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S || !drv[s].ranInner) return;
    InnerState& q = st[s];
    if (q.bestRes < q.finalResSum)
    {
        q.sel = q.best;
        q.finalResSum = q.bestRes;
    }
    else
    {
        q.sel = q.cur;
    }
}

__global__ void __launch_bounds__(NT) kb_mean_delta(BArgs B)
{
    CFB_TILE_BEGIN(t)
    if (!B.drv[s].ranInner || !B.drv[s].deflate) continue;
    double acc[1] = {0.0};
    CFB_ROWS acc[0] += (double)B.D[(size_t)B.st[s].sel * B.N + row];
    if (sys_sum<1>(acc, B, t, s, &B.drv[s].ticket) && threadIdx.x == 0)
        B.drv[s].dmean = acc[0] / (double)sy.n;
    CFB_TILE_END
}

__global__ void kb_psi_update(BArgs B)
{
    CFB_TILE_BEGIN(t)
    if (!B.drv[s].ranInner) continue;
    CFB_ROWS
    {
    const double m = B.drv[s].deflate ? B.drv[s].dmean : 0.0;
    const double dv = (double)B.D[(size_t)B.st[s].sel * B.N + row];
    B.psi[row] = __dadd_rn(B.psi[row], __dsub_rn(dv, m));
    }
    CFB_TILE_END
}

template <int MAXW>
__global__ void __launch_bounds__(NT) kb_residual(BArgs B)
{
    CFB_TILE_BEGIN(t)
    if (!B.drv[s].ranInner) continue;
    const bool deflate = B.drv[s].deflate;
    double acc[2] = {0.0, 0.0};
    CFB_ROWS
    {
        const double* psi = B.psi;
        const double wa = row_f64<MAXW>(B.A, B.A.val64, row, __dmul_rn(B.diag64[row], psi[row]),
                                        [&](int c) { return __ldg(psi + c); });
        const double rr = __dsub_rn(B.b[row], wa);
        B.r64[row] = rr;
        if (deflate)
        {
            const double uu = B.u[row];
            acc[0] += uu * rr;
            acc[1] += uu * uu;
        }
        else
        {
            acc[0] += fabs(rr);
        }
    }
    if (sys_sum<2>(acc, B, t, s, &B.drv[s].ticket) && threadIdx.x == 0)
    {
        BDrv& d = B.drv[s];
        if (deflate)
        {
            d.ur = acc[0];
            d.uu = acc[1];
        }
        else
        {
            d.finalRes = acc[0] / d.normFactor;
        }
    }
    CFB_TILE_END
}

__global__ void __launch_bounds__(NT) kb_cshift(BArgs B)
{
    CFB_TILE_BEGIN(t)
    if (!B.drv[s].ranInner || !B.drv[s].deflate) continue;
    const double ur = B.drv[s].ur;
    const double uu = B.drv[s].uu;
    const bool apply = uu > VSMALL;
    const double c = apply ? ur / uu : 0.0;
    double acc[1] = {0.0};
    CFB_ROWS
    {
        double rr = B.r64[row];
        if (apply)
        {
            B.psi[row] = __dadd_rn(B.psi[row], c);
            rr = __dsub_rn(rr, __dmul_rn(c, B.u[row]));
            B.r64[row] = rr;
        }
        acc[0] += fabs(rr);
    }
    if (sys_sum<1>(acc, B, t, s, &B.drv[s].ticket) && threadIdx.x == 0)
        B.drv[s].finalRes = acc[0] / B.drv[s].normFactor;
    CFB_TILE_END
}

// end of an outer pass (metalFoamSolver.C:313-414), per system
__global__ void kb_outer_end(int S, InnerState* st, BDrv* drv, int* counters, cf_options o,
                             int outer)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S) return;
    BDrv& d = drv[s];
    if (d.ranInner)
    {
        const InnerState& q = st[s];
        d.totalIter += q.it;
        d.singular = q.singular;
        d.stagnated = q.stagnated;
        d.finalResSum32 = q.finalResSum;
        if (d.deflate && d.finalRes > d.prevRes / 1.5 && !q.singular)
        {
            d.deflate = 0;
            d.polished = 1;
            d.restage = 1;
        }
        d.prevRes = d.finalRes;
        bool stop = false;
        if (d.singular) stop = true;
        if (d.totalIter >= o.maxIter) stop = true;
        if (d.totalIter >= o.minIter &&
            converged_(o.tolerance, o.relTol, d.initRes, d.finalRes))
            stop = true;
        if (stop)
        {
            d.finished = 1;
            d.nRestarts = outer;
        }
    }
    if (!d.finished) atomicAdd(&counters[1], 1);
}

__global__ void kb_unfinished_restarts(int S, BDrv* drv, int value)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < S && !drv[s].finished && drv[s].solved) drv[s].nRestarts = value;
}

__global__ void __launch_bounds__(NT) kb_l2(BArgs B)
{
    CFB_TILE_BEGIN(t)
    double acc[2] = {0.0, 0.0};
    CFB_ROWS
    {
        acc[0] += B.r64[row] * B.r64[row];
        acc[1] += B.b[row] * B.b[row];
    }
    if (sys_sum<2>(acc, B, t, s, &B.drv[s].ticket) && threadIdx.x == 0)
    {
        B.drv[s].l2r = sqrt(acc[0]);
        B.drv[s].l2b = sqrt(acc[1]);
    }
    CFB_TILE_END
}

}  // namespace

// ------------------------------------------------------------------ host side

struct cf_batch
{
    int device = 0;
    int numSMs = 1;
    int maxBlocksPerSM = 8;
    cudaStream_t ownStream = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    long long launches = 0;
    std::map<const void*, int> occ;
    bool finalized = false;
    bool coeffsDirty = true;

    struct Sys
    {
        int32_t n = 0, nf = 0;
        std::vector<int32_t> low, upp, own, los, losS;
        int32_t row0 = 0, npad = 0, tile0 = 0, ntiles = 0, face0 = 0;
        long long ent0 = 0;
        HostLayout L;
        bool hasCoeffs = false;
    };
    std::vector<Sys> sys;
    int S = 0;
    // systems that fill the GPU on their own run as single solves (one
    // context each, own stream) concurrently with the batched rest
    int32_t soloMinCells = 0;        // 0: automatic, < 0: never
    std::vector<cf_context*> solo;   // caller's index -> its context, or null
    std::vector<int> inner;          // caller's index -> index among the batched systems
    int nAll = 0;                    // systems as the caller numbers them
    long long N = 0, NF = 0, nnzp = 0;
    int nslices = 0, nTiles = 0;

    std::vector<void*> allocs;
    BSys* d_sys = nullptr;
    int2* d_tiles = nullptr;
    int* d_sliceOff = nullptr;
    int* d_col = nullptr;
    short* d_col16 = nullptr;   // row-relative 16-bit columns for the FP32 kernels, or null
    int* d_eface = nullptr;
    int* d_perm = nullptr;
    double *d_upper = nullptr, *d_diagIn = nullptr, *d_diag64 = nullptr, *d_u = nullptr;
    float* d_val32 = nullptr;
    double *d_val64 = nullptr, *d_valT64 = nullptr;
    float *d_diag32 = nullptr, *d_rD = nullptr;
    double *d_psi = nullptr, *d_b = nullptr, *d_r64 = nullptr, *d_io64 = nullptr,
           *d_io64b = nullptr;
    float *d_rA = nullptr, *d_W0 = nullptr, *d_W1 = nullptr, *d_Z0 = nullptr, *d_Z1 = nullptr,
          *d_P = nullptr, *d_Q = nullptr, *d_D = nullptr;
    InnerState* d_st = nullptr;
    BDrv* d_drv = nullptr;
    float* d_chebC = nullptr;
    double* d_part = nullptr;
    int* d_counters = nullptr;
    int* d_actTiles = nullptr;
    unsigned int* d_bar = nullptr;   // grid barrier of the persistent loop: count, gen, error
    bool coop = false;               // device supports cooperative launches
    BDrv* h_drv = nullptr;
    InnerState* h_st = nullptr;
    int* h_counters = nullptr;
    std::map<int, cudaGraphExec_t> graphs;
};

#define CFB_CUDA(call)                                                          \
    do                                                                          \
    {                                                                           \
        cudaError_t e_ = (call);                                                \
        if (e_ != cudaSuccess)                                                  \
            return fail(CF_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define CFB_TRY(expr)                 \
    do                                \
    {                                 \
        int rc_ = (expr);             \
        if (rc_ != CF_OK) return rc_; \
    } while (0)

#define CFB_LAUNCH()                                                            \
    do                                                                          \
    {                                                                           \
        cudaError_t e_ = cudaGetLastError();                                    \
        if (e_ != cudaSuccess)                                                  \
            return fail(CF_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e_)); \
        bt->launches++;                                                         \
    } while (0)

namespace {

template <class T>
int balloc(cf_batch* bt, T** p, size_t count)
{
    *p = nullptr;
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc((void**)p, count * sizeof(T));
    if (e != cudaSuccess) return fail(CF_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    bt->allocs.push_back((void*)*p);
    return CF_OK;
}

int bgrid(cf_batch* bt, const void* fn, long long work)
{
    int occ = 0;
    auto it = bt->occ.find(fn);
    if (it == bt->occ.end())
    {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, NT, 0) != cudaSuccess) occ = 1;
        occ = std::max(1, std::min(occ, bt->maxBlocksPerSM));
        bt->occ[fn] = occ;
    }
    else
    {
        occ = it->second;
    }
    const long long cap = (long long)bt->numSMs * occ;
    return (int)std::max(1LL, std::min(cap, work));
}

// tile kernels: work = tiles; row kernels: work = blocks of rows
int tgrid(cf_batch* bt, const void* fn) { return bgrid(bt, fn, bt->nTiles); }
int rgrid(cf_batch* bt, const void* fn) { return bgrid(bt, fn, (bt->N + NT - 1) / NT); }
int sgrid(cf_batch* bt) { return (bt->S + 127) / 128; }

BArgs bargs(const cf_batch* bt)
{
    BArgs B;
    B.nTiles = bt->nTiles;
    B.tiles = bt->d_tiles;
    B.sys = bt->d_sys;
    B.A.n = (int)bt->N;
    B.A.nslices = bt->nslices;
    B.A.sliceOff = bt->d_sliceOff;
    B.A.col = bt->d_col;
    B.A.col16 = bt->d_col16;
    B.A.val = bt->d_val32;
    B.A.val64 = bt->d_val64;
    B.N = bt->N;
    B.diag32 = bt->d_diag32;
    B.rD = bt->d_rD;
    B.chebC = bt->d_chebC;
    B.rA = bt->d_rA;
    B.W0 = bt->d_W0;
    B.W1 = bt->d_W1;
    B.Z0 = bt->d_Z0;
    B.Z1 = bt->d_Z1;
    B.P = bt->d_P;
    B.Q = bt->d_Q;
    B.D = bt->d_D;
    B.r64 = bt->d_r64;
    B.psi = bt->d_psi;
    B.b = bt->d_b;
    B.u = bt->d_u;
    B.diag64 = bt->d_diag64;
    B.st = bt->d_st;
    B.drv = bt->d_drv;
    B.part = bt->d_part;
    B.counters = bt->d_counters;
    B.actTiles = bt->d_actTiles;
    return B;
}

int launch_body(cf_batch* bt, int order, cudaGraphConditionalHandle h, int useCond)
{
    const BArgs B = bargs(bt);
    cudaStream_t s = bt->stream;
    const float* wA = B.W0;
    if (order > 1)
    {
        float* Z[2] = {B.Z0, B.Z1};
        for (int j = 1; j < order; ++j)
        {
            const float* zin = (j == 1) ? B.W0 : Z[(j - 1) & 1];
            const float* win = (j == 1) ? B.W0 : B.W1;
            if (j == order - 1)
            {
                auto fn = kb_cheb_step<true, MW>;
                fn<<<tgrid(bt, (const void*)fn), NT, 0, s>>>(B, zin, win, B.W1, Z[j & 1], j);
            }
            else
            {
                // one pass over up to 4 resident grids of sub-tiles: a batch
                // of small systems gets one row per thread, a batch whose
                // tiles would need many more blocks loops instead of
                // launching blocks that find no active tile
                const int g = (int)std::min<long long>((long long)bt->nTiles * kSubTiles,
                                                       4LL * bt->numSMs * bt->maxBlocksPerSM);
                kb_cheb_step_rows<MW><<<g, NT, 0, s>>>(B, zin, win, B.W1, Z[j & 1], j);
            }
            CFB_LAUNCH();
        }
        wA = Z[(order - 1) & 1];
    }
    {
        auto fn = kb_pcg_p_spmv<MW>;
        fn<<<tgrid(bt, (const void*)fn), NT, 0, s>>>(B, wA);
        CFB_LAUNCH();
    }
    if (order > 1)
    {
        auto fn = kb_pcg_update<true>;
        fn<<<tgrid(bt, (const void*)fn), NT, 0, s>>>(B, h, useCond);
    }
    else
    {
        auto fn = kb_pcg_update<false>;
        fn<<<tgrid(bt, (const void*)fn), NT, 0, s>>>(B, h, useCond);
    }
    CFB_LAUNCH();
    kb_compact<<<1, 1024, 0, s>>>(B, 0);
    CFB_LAUNCH();
    return CF_OK;
}

int batch_graph(cf_batch* bt, int order, cudaGraphExec_t* out)
{
    auto it = bt->graphs.find(order);
    if (it != bt->graphs.end())
    {
        *out = it->second;
        return CF_OK;
    }
    cudaGraph_t g = nullptr;
    CFB_CUDA(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle h;
    cudaError_t e = cudaGraphConditionalHandleCreate(&h, g, 1u, cudaGraphCondAssignDefault);
    if (e != cudaSuccess)
    {
        cudaGraphDestroy(g);
        return fail(CF_ERR_CUDA, std::string("cudaGraphConditionalHandleCreate: ") +
                                     cudaGetErrorString(e));
    }
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
        return fail(CF_ERR_CUDA, std::string("cudaGraphAddNode: ") + cudaGetErrorString(e));
    }
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    e = cudaStreamBeginCaptureToGraph(bt->stream, body, nullptr, nullptr, 0,
                                      cudaStreamCaptureModeRelaxed);
    if (e != cudaSuccess)
    {
        cudaGraphDestroy(g);
        return fail(CF_ERR_CUDA, std::string("cudaStreamBeginCaptureToGraph: ") +
                                     cudaGetErrorString(e));
    }
    const long long before = bt->launches;
    const int rc = launch_body(bt, order, h, 1);
    bt->launches = before;
    cudaGraph_t captured = nullptr;
    e = cudaStreamEndCapture(bt->stream, &captured);
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
    bt->graphs[order] = exec;
    *out = exec;
    return CF_OK;
}

// coefficients of every system -> device layout, row sums and census
int stage_batch(cf_batch* bt)
{
    cudaStream_t s = bt->stream;
    kb_gather<<<rgrid(bt, (const void*)kb_gather), NT, 0, s>>>(bt->N, bt->d_perm, bt->d_diagIn,
                                                               bt->d_diag64);
    CFB_LAUNCH();
    // symmetric FP32 operator (PCG); A^T values are not used by the batch
    const int g = bgrid(bt, (const void*)k_stage_vals, (bt->nnzp + NT - 1) / NT);
    k_stage_vals<<<g, NT, 0, s>>>(bt->nnzp, bt->d_col, bt->d_eface, bt->d_upper, bt->d_upper, 1,
                                  bt->d_val32, bt->d_val64, bt->d_valT64);
    CFB_LAUNCH();
    {
        auto fn = kb_sumA<MW>;
        fn<<<tgrid(bt, (const void*)fn), NT, 0, s>>>(bargs(bt));
        CFB_LAUNCH();
    }
    bt->coeffsDirty = false;
    return CF_OK;
}

bool converged_host(double tol, double relTol, double init, double fin)
{
    return (fin < tol) || (relTol > 1e-20 && fin < relTol * init);
}

int fetch_counters(cf_batch* bt)
{
    CFB_CUDA(cudaMemcpyAsync(bt->h_counters, bt->d_counters, 2 * sizeof(int),
                             cudaMemcpyDeviceToHost, bt->stream));
    CFB_CUDA(cudaStreamSynchronize(bt->stream));
    return CF_OK;
}

// The inner loop of all systems as one cooperative launch (kbp_pcg) when
// the device supports it; *ran tells whether it ran.  Waits for the launch
// and reports a grid barrier that gave up as CF_ERR_DEVICE_TIMEOUT.
int persistent_loop(cf_batch* bt, int order, bool* ran)
{
    *ran = false;
    if (!bt->coop) return CF_OK;
    const void* fn = order > 1 ? (const void*)kbp_pcg<true, MW> : (const void*)kbp_pcg<false, MW>;
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, NT, 0) != cudaSuccess || occ < 1)
    {
        cudaGetLastError();
        return CF_OK;
    }
    const int grid = (int)std::max(1LL, std::min((long long)occ * bt->numSMs,
                                                 (long long)bt->nTiles));
    cudaStream_t s = bt->stream;
    CFB_CUDA(cudaMemsetAsync(bt->d_bar, 0, sizeof(unsigned int) * 4, s));
    BArgs B = bargs(bt);
    GridBar bar{bt->d_bar, bt->d_bar + 1, reinterpret_cast<int*>(bt->d_bar + 2), 1ull << 24};
    int ord = order;
    void* args[] = {(void*)&B, (void*)&ord, (void*)&bar};
    const cudaError_t e = cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(NT), args, 0, s);
    if (e != cudaSuccess)
        return fail(CF_ERR_CUDA, std::string("cudaLaunchCooperativeKernel: ") + cudaGetErrorString(e));
    bt->launches++;
    int err = 0;
    CFB_CUDA(cudaMemcpyAsync(&err, bt->d_bar + 2, sizeof(int), cudaMemcpyDeviceToHost, s));
    CFB_CUDA(cudaStreamSynchronize(s));
    if (err) return fail(CF_ERR_DEVICE_TIMEOUT, "a grid barrier of the persistent batched loop timed out");
    *ran = true;
    return CF_OK;
}

int batch_solve(cf_batch* bt, double* const* psi, const double* const* src, bool hostPtrs,
                const cf_options* o, cf_performance* perf)
{
    cudaStream_t s = bt->stream;
    const cudaMemcpyKind in = hostPtrs ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    const cudaMemcpyKind out = hostPtrs ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    CFB_CUDA(cudaEventRecord(bt->ev0, s));
    for (int i = 0; i < bt->S; ++i)
    {
        const auto& y = bt->sys[i];
        CFB_CUDA(cudaMemcpyAsync(bt->d_io64 + y.row0, psi[i], sizeof(double) * y.n, in, s));
        CFB_CUDA(cudaMemcpyAsync(bt->d_io64b + y.row0, src[i], sizeof(double) * y.n, in, s));
    }
    if (bt->coeffsDirty) CFB_TRY(stage_batch(bt));
    const BArgs B = bargs(bt);
    const int gr = rgrid(bt, (const void*)kb_gather);
    kb_gather<<<gr, NT, 0, s>>>(bt->N, bt->d_perm, bt->d_io64, bt->d_psi);
    CFB_LAUNCH();
    kb_gather<<<gr, NT, 0, s>>>(bt->N, bt->d_perm, bt->d_io64b, bt->d_b);
    CFB_LAUNCH();
    kb_mean<0><<<tgrid(bt, (const void*)kb_mean<0>), NT, 0, s>>>(B);
    CFB_LAUNCH();
    {
        auto fn = kb_residual0<MW>;
        fn<<<tgrid(bt, (const void*)fn), NT, 0, s>>>(B);
        CFB_LAUNCH();
    }
    kb_entry<<<sgrid(bt), 128, 0, s>>>(bt->S, bt->d_drv, *o);
    CFB_LAUNCH();
    kb_entry_auto<<<sgrid(bt), 128, 0, s>>>(bt->S, bt->d_sys, bt->d_drv, o->deflate);
    CFB_LAUNCH();
    kb_stage_diag32<<<tgrid(bt, (const void*)kb_stage_diag32), NT, 0, s>>>(B, bt->d_diag32,
                                                                          bt->d_rD, 0);
    CFB_LAUNCH();
    const int order = o->chebyshevOrder;
    if (order > 1)
    {
        auto fn = kb_gershgorin<MW>;
        fn<<<tgrid(bt, (const void*)fn), NT, 0, s>>>(B, bt->d_eface, bt->d_upper, order,
                                                    o->chebyshevRatio, bt->d_chebC);
        CFB_LAUNCH();
    }
    int outer = 0;
    bool all_done = false;
    for (outer = 0; outer <= o->maxRestarts; ++outer)
    {
        CFB_CUDA(cudaMemsetAsync(bt->d_counters, 0, 2 * sizeof(int), s));
        kb_outer_begin<<<sgrid(bt), 128, 0, s>>>(bt->S, bt->d_st, bt->d_drv, bt->d_counters,
                                                 o->maxIter, o->iterationsPerSync,
                                                 o->stagnationLimit);
        CFB_LAUNCH();
        kb_mean<1><<<tgrid(bt, (const void*)kb_mean<1>), NT, 0, s>>>(B);
        CFB_LAUNCH();
        if (order > 1)
            kb_pcg_init<true><<<tgrid(bt, (const void*)kb_pcg_init<true>), NT, 0, s>>>(B);
        else
            kb_pcg_init<false><<<tgrid(bt, (const void*)kb_pcg_init<false>), NT, 0, s>>>(B);
        CFB_LAUNCH();
        kb_compact<<<1, 1024, 0, s>>>(B, 1);
        CFB_LAUNCH();
        CFB_TRY(fetch_counters(bt));
        if (bt->h_counters[0] > 0)
        {
            // opt-in: the whole inner loop of all systems as one launch
            bool ran = false;
            if (o->graph && o->persistentMaxCells > 0 && bt->N <= o->persistentMaxCells)
                CFB_TRY(persistent_loop(bt, order, &ran));
            if (!ran && o->graph)
            {
                cudaGraphExec_t exec;
                CFB_TRY(batch_graph(bt, order, &exec));
                CFB_CUDA(cudaGraphLaunch(exec, s));
            }
            else if (!ran)
            {
                for (int it = 0; it < o->maxIter; ++it)
                {
                    CFB_TRY(launch_body(bt, order, 0, 0));
                    CFB_TRY(fetch_counters(bt));
                    if (bt->h_counters[0] <= 0) break;
                }
            }
        }
        kb_inner_final<<<sgrid(bt), 128, 0, s>>>(bt->S, bt->d_st, bt->d_drv);
        CFB_LAUNCH();
        kb_mean_delta<<<tgrid(bt, (const void*)kb_mean_delta), NT, 0, s>>>(B);
        CFB_LAUNCH();
        kb_psi_update<<<tgrid(bt, (const void*)kb_psi_update), NT, 0, s>>>(B);
        CFB_LAUNCH();
        {
            auto fn = kb_residual<MW>;
            fn<<<tgrid(bt, (const void*)fn), NT, 0, s>>>(B);
            CFB_LAUNCH();
        }
        kb_cshift<<<tgrid(bt, (const void*)kb_cshift), NT, 0, s>>>(B);
        CFB_LAUNCH();
        CFB_CUDA(cudaMemsetAsync(bt->d_counters + 1, 0, sizeof(int), s));
        kb_outer_end<<<sgrid(bt), 128, 0, s>>>(bt->S, bt->d_st, bt->d_drv, bt->d_counters, *o,
                                               outer);
        CFB_LAUNCH();
        kb_stage_diag32<<<tgrid(bt, (const void*)kb_stage_diag32), NT, 0, s>>>(B, bt->d_diag32,
                                                                              bt->d_rD, 1);
        CFB_LAUNCH();
        CFB_TRY(fetch_counters(bt));
        if (bt->h_counters[1] == 0)
        {
            all_done = true;
            break;
        }
    }
    if (!all_done)
    {
        kb_unfinished_restarts<<<sgrid(bt), 128, 0, s>>>(bt->S, bt->d_drv, o->maxRestarts + 1);
        CFB_LAUNCH();
    }
    kb_l2<<<tgrid(bt, (const void*)kb_l2), NT, 0, s>>>(B);
    CFB_LAUNCH();
    kb_scatter<<<gr, NT, 0, s>>>(bt->N, bt->d_perm, bt->d_psi, bt->d_io64);
    CFB_LAUNCH();
    for (int i = 0; i < bt->S; ++i)
    {
        const auto& y = bt->sys[i];
        CFB_CUDA(cudaMemcpyAsync(psi[i], bt->d_io64 + y.row0, sizeof(double) * y.n, out, s));
    }
    CFB_CUDA(cudaEventRecord(bt->ev1, s));
    CFB_CUDA(cudaMemcpyAsync(bt->h_drv, bt->d_drv, sizeof(BDrv) * bt->S, cudaMemcpyDeviceToHost,
                             s));
    CFB_CUDA(cudaStreamSynchronize(s));
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, bt->ev0, bt->ev1);
    for (int i = 0; i < bt->S; ++i)
    {
        const BDrv& d = bt->h_drv[i];
        cf_performance& p = perf[i];
        std::memset(&p, 0, sizeof(p));
        p.initialResidual = d.initRes;
        p.finalResidual = d.finalRes;
        p.nIterations = d.totalIter;
        p.nRestarts = d.nRestarts;
        p.converged = converged_host(o->tolerance, o->relTol, d.initRes, d.finalRes);
        p.singular = d.singular;
        p.stagnated = d.stagnated;
        p.deflated = d.deflate || d.polished;
        p.polished = d.polished;
        p.solved = d.solved;
        p.normFactor = d.normFactor;
        p.chebBeta = order > 1 ? d.chebBeta : 2.0;
        p.finalResSum32 = d.finalResSum32;
        p.residualL2 = d.l2b > 0 ? d.l2r / d.l2b : d.l2r;
        p.tSolve = ms * 1e-3;
    }
    return CF_OK;
}

}  // namespace

// ------------------------------------------------------------------ C ABI

extern "C" int cf_batch_create(cf_batch** out, int32_t device)
{
    if (!out) return fail(CF_ERR_INVALID_ARG, "out is NULL");
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
    {
        cudaGetLastError();
        return fail(CF_ERR_NO_DEVICE, "cudaFoam: no CUDA device available");
    }
    if (device < 0 || device >= count) return fail(CF_ERR_INVALID_ARG, "device out of range");
    cudaDeviceProp prop;
    CFB_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10)
        return fail(CF_ERR_NO_DEVICE, std::string("cudaFoam: ") + prop.name +
                                          " is not an sm_100 (B200-class) device");
    CFB_CUDA(cudaSetDevice(device));
    cf_batch* bt = new cf_batch();
    bt->device = device;
    bt->numSMs = prop.multiProcessorCount;
    bt->maxBlocksPerSM = std::max(1, prop.maxThreadsPerMultiProcessor / NT);
    bt->coop = prop.cooperativeLaunch != 0;
    if (cudaStreamCreateWithFlags(&bt->ownStream, cudaStreamNonBlocking) != cudaSuccess)
    {
        delete bt;
        return fail(CF_ERR_CUDA, "cudaStreamCreate failed");
    }
    bt->stream = bt->ownStream;
    cudaEventCreate(&bt->ev0);
    cudaEventCreate(&bt->ev1);
    *out = bt;
    return CF_OK;
}

extern "C" int cf_batch_destroy(cf_batch* bt)
{
    if (!bt) return CF_OK;
    cudaSetDevice(bt->device);
    if (bt->stream) cudaStreamSynchronize(bt->stream);
    for (cf_context* c : bt->solo)
        if (c) cf_context_destroy(c);
    for (auto& kv : bt->graphs) cudaGraphExecDestroy(kv.second);
    for (void* p : bt->allocs) cudaFree(p);
    if (bt->h_drv) cudaFreeHost(bt->h_drv);
    if (bt->h_st) cudaFreeHost(bt->h_st);
    if (bt->h_counters) cudaFreeHost(bt->h_counters);
    if (bt->ev0) cudaEventDestroy(bt->ev0);
    if (bt->ev1) cudaEventDestroy(bt->ev1);
    if (bt->ownStream) cudaStreamDestroy(bt->ownStream);
    delete bt;
    return CF_OK;
}

extern "C" int cf_batch_set_stream(cf_batch* bt, void* stream)
{
    if (!bt) return fail(CF_ERR_INVALID_ARG, "batch is NULL");
    bt->stream = stream ? (cudaStream_t)stream : bt->ownStream;
    return CF_OK;
}

extern "C" int cf_batch_kernel_launches(const cf_batch* bt, long long* count)
{
    if (!bt || !count) return fail(CF_ERR_INVALID_ARG, "NULL argument");
    long long n = bt->launches;
    for (const cf_context* c : bt->solo)
    {
        long long k = 0;
        if (c && cf_context_kernel_launches(c, &k) == CF_OK) n += k;
    }
    *count = n;
    return CF_OK;
}

extern "C" int cf_batch_add_system(cf_batch* bt, int32_t n, int32_t nf, const int32_t* low,
                                   const int32_t* upp, const int32_t* own, const int32_t* los,
                                   const int32_t* losS, int32_t* index)
{
    if (!bt) return fail(CF_ERR_INVALID_ARG, "batch is NULL");
    if (bt->finalized) return fail(CF_ERR_INVALID_ARG, "batch already finalised");
    if (n <= 0 || nf < 0) return fail(CF_ERR_INVALID_ARG, "nCells must be > 0, nFaces >= 0");
    if ((nf > 0 && (!low || !upp || !los)) || !own || !losS)
        return fail(CF_ERR_INVALID_ARG, "NULL addressing array");
    CFB_TRY(check_addressing(n, nf, low, upp, own, los, losS));
    cf_batch::Sys y;
    y.n = n;
    y.nf = nf;
    y.low.assign(low, low + nf);
    y.upp.assign(upp, upp + nf);
    y.own.assign(own, own + n + 1);
    y.los.assign(los, los + nf);
    y.losS.assign(losS, losS + n + 1);
    bt->sys.push_back(std::move(y));
    if (index) *index = (int32_t)bt->sys.size() - 1;
    return CF_OK;
}

extern "C" int cf_batch_finalize(cf_batch* bt, int32_t reorder)
{
    if (!bt) return fail(CF_ERR_INVALID_ARG, "batch is NULL");
    if (bt->finalized) return CF_OK;
    if (bt->sys.empty()) return fail(CF_ERR_INVALID_ARG, "batch has no systems");
    CFB_CUDA(cudaSetDevice(bt->device));
    // systems of at least three blocks of rows per SM become solo systems:
    // their single solves keep the GPU busy beside the others, while the
    // small ones run their iterations as one launch per phase for all
    // (measured on the 48-system set: 8 solo systems from numSMs x 2048
    // rows, 588 ms; 17-19 from 3 x 256 per SM or 100,000, 545 ms)
    {
        const long long minCells =
            bt->soloMinCells > 0 ? bt->soloMinCells
                                 : (bt->soloMinCells == 0 ? (long long)bt->numSMs * SOLO_BLOCKS_PER_SM * NT
                                                          : (1LL << 62));
        bt->nAll = (int)bt->sys.size();
        bt->solo.assign(bt->nAll, nullptr);
        bt->inner.assign(bt->nAll, -1);
        std::vector<cf_batch::Sys> keep;
        for (int i = 0; i < bt->nAll; ++i)
        {
            auto& y = bt->sys[i];
            if ((long long)y.n < minCells)
            {
                bt->inner[i] = (int)keep.size();
                keep.push_back(std::move(y));
                continue;
            }
            cf_context* c = nullptr;
            CFB_TRY(cf_context_create(&c, bt->device));
            bt->solo[i] = c;
            CFB_TRY(cf_context_set_reorder(c, reorder));
            CFB_TRY(cf_set_topology(c, y.n, y.nf, y.low.data(), y.upp.data(), y.own.data(),
                                    y.los.data(), y.losS.data()));
        }
        bt->sys.swap(keep);
        if (bt->sys.empty())
        {
            bt->S = 0;
            bt->finalized = true;
            return CF_OK;
        }
    }
    bt->S = (int)bt->sys.size();
    long long row = 0, face = 0, ent = 0;
    int tile = 0, slices = 0;
    std::vector<BSys> hs(bt->S);
    std::vector<int2> tiles;
    for (int i = 0; i < bt->S; ++i)
    {
        auto& y = bt->sys[i];
        const bool rcm = reorder == CF_REORDER_RCM || (reorder == CF_REORDER_AUTO && y.n > 65536);
        CFB_TRY(build_layout(y.n, y.nf, y.low.data(), y.upp.data(), y.own.data(), y.los.data(),
                             y.losS.data(), rcm, y.L));
        y.row0 = (int32_t)row;
        y.npad = y.L.nslices * SLICE;
        y.face0 = (int32_t)face;
        y.ent0 = ent;
        y.tile0 = tile;
        y.ntiles = (y.npad + kTileRows - 1) / kTileRows;
        for (int k = 0; k < y.ntiles; ++k) tiles.push_back(make_int2(i, y.row0 + k * kTileRows));
        hs[i] = BSys{y.row0, y.n, y.npad, y.tile0, y.ntiles, y.face0, y.nf};
        row += y.npad;
        face += y.nf;
        ent += y.L.nnzp;
        tile += y.ntiles;
        slices += y.L.nslices;
        if (row >= (1LL << 31) - 1024 || ent >= (1LL << 31) - 64)
            return fail(CF_ERR_TOO_LARGE, "batch too large for 32-bit row/entry offsets");
    }
    bt->N = row;
    bt->NF = face;
    bt->nnzp = ent;
    bt->nTiles = tile;
    bt->nslices = slices;
    // concatenated layout
    std::vector<int32_t> sliceOff(slices + 1, 0), col(std::max(ent, 1LL), -1),
        eface(std::max(ent, 1LL), -1), perm(row, -1);
    int sl = 0;
    for (int i = 0; i < bt->S; ++i)
    {
        const auto& y = bt->sys[i];
        for (int k = 0; k < y.L.nslices; ++k) sliceOff[sl + k] = (int32_t)(y.ent0 + y.L.sliceOff[k]);
        sl += y.L.nslices;
        for (long long e = 0; e < y.L.nnzp; ++e)
        {
            const int32_t c = y.L.col[e];
            if (c == -1) continue;
            const uint32_t idx = ((uint32_t)c & 0x7fffffffu) + (uint32_t)y.row0;
            col[y.ent0 + e] = (int32_t)(idx | ((uint32_t)c & 0x80000000u));
            eface[y.ent0 + e] = y.L.eface[e] + y.face0;
        }
        for (int32_t r = 0; r < y.n; ++r) perm[y.row0 + r] = y.row0 + y.L.perm[r];
    }
    sliceOff[slices] = (int32_t)ent;
    // compact column stream of the FP32 kernels (as for one system: the same
    // columns as row-relative 16-bit offsets, when every system's columns lie
    // within 32767 rows of their row; each system starts on a slice boundary,
    // so slice k of the concatenation holds global rows 32 k .. 32 k + 31)
    std::vector<short> col16;
    {
        bool fits = true;
        std::vector<short> c16((size_t)std::max(ent, 1LL), COL16_PAD);
        for (int k = 0; k < slices && fits; ++k)
        {
            const int32_t w = (sliceOff[k + 1] - sliceOff[k]) / SLICE;
            for (int32_t j = 0; j < w && fits; ++j)
                for (int32_t l = 0; l < SLICE; ++l)
                {
                    const long long e = (long long)sliceOff[k] + (long long)SLICE * j + l;
                    if (col[e] == -1) continue;
                    const long long off = (long long)((uint32_t)col[e] & 0x7fffffffu) -
                                          ((long long)k * SLICE + l);
                    if (off < -32767 || off > 32767)
                    {
                        fits = false;
                        break;
                    }
                    c16[e] = (short)off;
                }
        }
        if (fits) col16.swap(c16);
    }
    const size_t N = (size_t)row;
    CFB_TRY(balloc(bt, &bt->d_sys, bt->S));
    CFB_TRY(balloc(bt, &bt->d_tiles, (size_t)tile));
    CFB_TRY(balloc(bt, &bt->d_sliceOff, (size_t)slices + 1));
    CFB_TRY(balloc(bt, &bt->d_col, col.size()));
    CFB_TRY(balloc(bt, &bt->d_eface, eface.size()));
    CFB_TRY(balloc(bt, &bt->d_perm, N));
    CFB_TRY(balloc(bt, &bt->d_upper, (size_t)std::max(face, 1LL)));
    CFB_TRY(balloc(bt, &bt->d_diagIn, N));
    CFB_TRY(balloc(bt, &bt->d_diag64, N));
    CFB_TRY(balloc(bt, &bt->d_u, N));
    CFB_TRY(balloc(bt, &bt->d_val32, col.size()));
    CFB_TRY(balloc(bt, &bt->d_val64, col.size()));
    CFB_TRY(balloc(bt, &bt->d_valT64, col.size()));
    CFB_TRY(balloc(bt, &bt->d_diag32, N));
    CFB_TRY(balloc(bt, &bt->d_rD, N));
    CFB_TRY(balloc(bt, &bt->d_psi, N));
    CFB_TRY(balloc(bt, &bt->d_b, N));
    CFB_TRY(balloc(bt, &bt->d_r64, N));
    CFB_TRY(balloc(bt, &bt->d_io64, N));
    CFB_TRY(balloc(bt, &bt->d_io64b, N));
    CFB_TRY(balloc(bt, &bt->d_rA, N));
    CFB_TRY(balloc(bt, &bt->d_W0, N));
    CFB_TRY(balloc(bt, &bt->d_W1, N));
    CFB_TRY(balloc(bt, &bt->d_Z0, N));
    CFB_TRY(balloc(bt, &bt->d_Z1, N));
    CFB_TRY(balloc(bt, &bt->d_P, 2 * N));
    CFB_TRY(balloc(bt, &bt->d_Q, N));
    CFB_TRY(balloc(bt, &bt->d_D, 3 * N));
    CFB_TRY(balloc(bt, &bt->d_st, bt->S));
    CFB_TRY(balloc(bt, &bt->d_drv, bt->S));
    CFB_TRY(balloc(bt, &bt->d_chebC, (size_t)bt->S * kChebStride));
    CFB_TRY(balloc(bt, &bt->d_part, (size_t)NPART * tile));
    CFB_TRY(balloc(bt, &bt->d_counters, 4));
    CFB_TRY(balloc(bt, &bt->d_actTiles, (size_t)tile));
    CFB_TRY(balloc(bt, &bt->d_bar, 4));
    CFB_CUDA(cudaMallocHost((void**)&bt->h_drv, sizeof(BDrv) * bt->S));
    CFB_CUDA(cudaMallocHost((void**)&bt->h_st, sizeof(InnerState) * bt->S));
    CFB_CUDA(cudaMallocHost((void**)&bt->h_counters, 4 * sizeof(int)));
    cudaStream_t s = bt->stream;
    CFB_CUDA(cudaMemcpyAsync(bt->d_sys, hs.data(), sizeof(BSys) * bt->S, cudaMemcpyHostToDevice, s));
    CFB_CUDA(cudaMemcpyAsync(bt->d_tiles, tiles.data(), sizeof(int2) * tile, cudaMemcpyHostToDevice, s));
    CFB_CUDA(cudaMemcpyAsync(bt->d_sliceOff, sliceOff.data(), sizeof(int32_t) * sliceOff.size(),
                             cudaMemcpyHostToDevice, s));
    CFB_CUDA(cudaMemcpyAsync(bt->d_col, col.data(), sizeof(int32_t) * col.size(),
                             cudaMemcpyHostToDevice, s));
    if (!col16.empty())
    {
        CFB_TRY(balloc(bt, &bt->d_col16, col16.size()));
        CFB_CUDA(cudaMemcpyAsync(bt->d_col16, col16.data(), sizeof(short) * col16.size(),
                                 cudaMemcpyHostToDevice, s));
    }
    CFB_CUDA(cudaMemcpyAsync(bt->d_eface, eface.data(), sizeof(int32_t) * eface.size(),
                             cudaMemcpyHostToDevice, s));
    CFB_CUDA(cudaMemcpyAsync(bt->d_perm, perm.data(), sizeof(int32_t) * N, cudaMemcpyHostToDevice, s));
    CFB_CUDA(cudaMemsetAsync(bt->d_st, 0, sizeof(InnerState) * bt->S, s));
    CFB_CUDA(cudaMemsetAsync(bt->d_drv, 0, sizeof(BDrv) * bt->S, s));
    CFB_CUDA(cudaMemsetAsync(bt->d_counters, 0, 4 * sizeof(int), s));
    CFB_CUDA(cudaMemsetAsync(bt->d_diagIn, 0, sizeof(double) * N, s));
    CFB_CUDA(cudaMemsetAsync(bt->d_D, 0, sizeof(float) * 3 * N, s));
    CFB_CUDA(cudaMemsetAsync(bt->d_io64, 0, sizeof(double) * N, s));
    CFB_CUDA(cudaMemsetAsync(bt->d_io64b, 0, sizeof(double) * N, s));
    CFB_CUDA(cudaStreamSynchronize(s));
    for (auto& y : bt->sys)
    {
        std::vector<int32_t>().swap(y.L.col);   // host copies no longer needed
        std::vector<int32_t>().swap(y.L.eface);
    }
    bt->finalized = true;
    return CF_OK;
}

static int batch_set_coeffs(cf_batch* bt, int32_t i, const double* diag, const double* upper,
                            const double* lower, cudaMemcpyKind kind)
{
    if (!bt || !bt->finalized) return fail(CF_ERR_INVALID_ARG, "batch not finalised");
    if (i < 0 || i >= bt->nAll) return fail(CF_ERR_INVALID_ARG, "system index out of range");
    if (lower) return fail(CF_ERR_UNSUPPORTED, "batched solves take symmetric matrices (PCG)");
    if (bt->solo[i])
    {
        if (kind == cudaMemcpyHostToDevice)
            return cf_set_coeffs(bt->solo[i], diag, upper, nullptr, nullptr);
        // device data: ordered after the batch stream's earlier work
        CFB_CUDA(cudaStreamSynchronize(bt->stream));
        return cf_set_coeffs_device(bt->solo[i], diag, upper, nullptr);
    }
    i = bt->inner[i];
    const auto& y = bt->sys[i];
    if (!diag || (y.nf > 0 && !upper)) return fail(CF_ERR_INVALID_ARG, "NULL coefficient array");
    CFB_CUDA(cudaSetDevice(bt->device));
    CFB_CUDA(cudaMemcpyAsync(bt->d_diagIn + y.row0, diag, sizeof(double) * y.n, kind, bt->stream));
    if (y.nf > 0)
        CFB_CUDA(cudaMemcpyAsync(bt->d_upper + y.face0, upper, sizeof(double) * y.nf, kind,
                                 bt->stream));
    bt->sys[i].hasCoeffs = true;
    bt->coeffsDirty = true;
    return CF_OK;
}

extern "C" int cf_batch_set_coeffs(cf_batch* bt, int32_t i, const double* diag,
                                   const double* upper, const double* lower)
{
    return batch_set_coeffs(bt, i, diag, upper, lower, cudaMemcpyHostToDevice);
}

extern "C" int cf_batch_set_coeffs_device(cf_batch* bt, int32_t i, const double* diag,
                                          const double* upper, const double* lower)
{
    return batch_set_coeffs(bt, i, diag, upper, lower, cudaMemcpyDeviceToDevice);
}

static int batch_check(cf_batch* bt, int32_t solver, const cf_options* o, cf_performance* perf,
                       const void* psi, const void* src)
{
    if (!bt || !bt->finalized) return fail(CF_ERR_INVALID_ARG, "batch not finalised");
    if (solver != CF_SOLVER_PCG)
        return fail(CF_ERR_UNSUPPORTED, "batched solves are cudaPCG (symmetric pressure systems)");
    if (!o || !perf || !psi || !src) return fail(CF_ERR_INVALID_ARG, "NULL argument");
    if (o->preconditioner != CF_PRECOND_CHEBYSHEV)
        return fail(CF_ERR_UNSUPPORTED, "batched solves use the Chebyshev-Jacobi preconditioner "
                                        "(GAMG systems: one context each, cf_solve_many_device)");
    if (o->chebyshevOrder < 1 || o->chebyshevOrder > CF_MAX_CHEB)
        return fail(CF_ERR_INVALID_ARG, "chebyshevOrder must be in [1, 64]");
    if (o->deflate < CF_DEFLATE_AUTO || o->deflate > CF_DEFLATE_OFF)
        return fail(CF_ERR_INVALID_ARG, "bad deflate option");
    if (!(o->chebyshevRatio > 1.0)) return fail(CF_ERR_INVALID_ARG, "chebyshevRatio must be > 1");
    for (const auto& y : bt->sys)
        if (!y.hasCoeffs) return fail(CF_ERR_NO_COEFFS, "a system has no coefficients");
    CFB_CUDA(cudaSetDevice(bt->device));
    return CF_OK;
}

// The batched systems through batch_solve on the calling thread, each solo
// system through cf_solve[_device] on a thread and stream of its own, all at
// once; every system gets what its own path returns.
static int batch_solve_all(cf_batch* bt, double* const* psi, const double* const* src,
                           bool hostPtrs, const cf_options* o, cf_performance* perf)
{
    std::vector<double*> ip;
    std::vector<const double*> is;
    std::vector<int> solos;
    for (int i = 0; i < bt->nAll; ++i)
    {
        if (bt->solo[i])
        {
            solos.push_back(i);
        }
        else
        {
            ip.push_back(psi[i]);
            is.push_back(src[i]);
        }
    }
    if (!solos.empty() && !hostPtrs) CFB_CUDA(cudaStreamSynchronize(bt->stream));
    std::vector<int> rc(bt->nAll, CF_OK);
    std::vector<std::string> msg(bt->nAll);
    auto run = [&](int i) {
        const int r = hostPtrs ? cf_solve(bt->solo[i], CF_SOLVER_PCG, psi[i], src[i], o, &perf[i])
                               : cf_solve_device(bt->solo[i], CF_SOLVER_PCG, psi[i], src[i], o,
                                                 &perf[i]);
        if (r != CF_OK) msg[i] = cf_last_error();
        rc[i] = r;
    };
    std::vector<std::thread> pool;
    std::vector<int> inlineRuns;
    for (int i : solos)
    {
        try
        {
            pool.emplace_back(run, i);
        }
        catch (...)
        {
            inlineRuns.push_back(i);   // no exception crosses the C ABI
        }
    }
    int brc = CF_OK;
    std::string bmsg;
    if (bt->S > 0)
    {
        std::vector<cf_performance> bp(bt->S);
        brc = batch_solve(bt, ip.data(), is.data(), hostPtrs, o, bp.data());
        if (brc != CF_OK)
            bmsg = cf_last_error();
        else
            for (int i = 0; i < bt->nAll; ++i)
                if (!bt->solo[i]) perf[i] = bp[bt->inner[i]];
    }
    for (int i : inlineRuns) run(i);
    for (auto& t : pool) t.join();
    if (brc != CF_OK) return fail(brc, bmsg);
    for (int i : solos)
        if (rc[i] != CF_OK) return fail(rc[i], "system " + std::to_string(i) + ": " + msg[i]);
    return CF_OK;
}

extern "C" int cf_batch_solve(cf_batch* bt, int32_t solver, double* const* psi,
                              const double* const* source, const cf_options* o,
                              cf_performance* perf)
{
    CFB_TRY(batch_check(bt, solver, o, perf, psi, source));
    return batch_solve_all(bt, psi, source, true, o, perf);
}

extern "C" int cf_batch_solve_device(cf_batch* bt, int32_t solver, double* const* psi,
                                     const double* const* source, const cf_options* o,
                                     cf_performance* perf)
{
    CFB_TRY(batch_check(bt, solver, o, perf, psi, source));
    return batch_solve_all(bt, psi, source, false, o, perf);
}

extern "C" int cf_batch_set_solo_cells(cf_batch* bt, int32_t minCells)
{
    if (!bt) return fail(CF_ERR_INVALID_ARG, "batch is NULL");
    if (bt->finalized) return fail(CF_ERR_INVALID_ARG, "batch already finalised");
    bt->soloMinCells = minCells;
    return CF_OK;
}
