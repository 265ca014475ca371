// cf_kernels.cuh -- sm_100a kernels of the Krylov hot path.
//
// The reference runs 14 small MSL kernels per iteration family with a
// single-threadgroup scalar pass after every reduction
// (src/metal4Foam/shaders/metalFoamKernels.metal, dispatch sequences in
// src/metal4Foam/backend/metalFoamBackend.C:608-906).  Here:
//
//  * every reduction is finished inside the kernel that produces it: each
//    block writes one FP64 partial, the last block to arrive (atomic
//    ticket, no spin) folds the partials in a fixed order and updates the
//    solver scalars (alpha, beta, omega, residual, convergence flags);
//  * dot and L1 partials accumulate the FP32 products in FP64 (exact
//    products, FP64 sums) -- the compensated reductions of the design;
//  * the vector updates are fused with their neighbours: Chebyshev step =
//    SpMV + recurrence (+ the z.r dot on the last step), p-update fused into
//    the SpMV's x-gather, solution/residual update fused with the L1 partial
//    and the next preconditioner apply (and its dot);
//  * one kernel per phase, captured once into a CUDA graph whose
//    conditional WHILE node runs the iterations on the device.
//
// All FP32 arithmetic that the reference kernels do element-wise uses
// explicitly rounded intrinsics (__fmul_rn/__fadd_rn/__fsub_rn) so nothing
// is contracted into an FMA: the per-element results are bit-identical to
// the reference kernels' source semantics given the same scalars.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "cf_internal.cuh"

namespace cf {

// ----------------------------------------------------------------- helpers

__host__ __device__ inline void cheb_constants(int order, double beta,
                                               double ratio, float* c)
{
    // encCheb (metalFoamBackend.C:342-385): spectrum [beta/ratio, beta] of
    // rD*A; c[0] = c1, (c2, c3) of step i at c[2i-1], c[2i].
    const double alpha = beta / ratio;
    const double theta = 0.5 * (beta + alpha);
    const double delta = 0.5 * (beta - alpha);
    const double sigma = theta / delta;
    double rho = 1.0 / sigma;
    c[0] = (float)(1.0 / theta);
    for (int i = 1; i < order; ++i)
    {
        const double rhoNew = 1.0 / (2.0 * sigma - rho);
        c[2 * i - 1] = (float)(rhoNew * rho);
        c[2 * i] = (float)(2.0 * rhoNew / delta);
        rho = rhoNew;
    }
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double warp_max(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Block sum of NR values; totals valid in warp 0.
template <int NR>
__device__ __forceinline__ void block_sum(double (&v)[NR])
{
    __shared__ double sh[NR][NT / 32];
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    __syncthreads();
#pragma unroll
    for (int r = 0; r < NR; ++r) v[r] = warp_sum(v[r]);
    if (lane == 0)
    {
#pragma unroll
        for (int r = 0; r < NR; ++r) sh[r][wid] = v[r];
    }
    __syncthreads();
    if (wid == 0)
    {
#pragma unroll
        for (int r = 0; r < NR; ++r)
        {
            double t = lane < NT / 32 ? sh[r][lane] : 0.0;
            v[r] = warp_sum(t);
        }
    }
}

// Grid-wide sum of NR values per thread.  Returns true in the last block to
// finish; its thread 0 then holds the totals in v (summed in an order that
// depends only on gridDim, so results are reproducible) and must finalise.
template <int NR>
__device__ __forceinline__ bool grid_sum(double (&v)[NR], double* part,
                                         unsigned int* ticket)
{
    __shared__ bool amLast;
    block_sum<NR>(v);
    if (threadIdx.x == 0)
    {
#pragma unroll
        for (int r = 0; r < NR; ++r) part[r * gridDim.x + blockIdx.x] = v[r];
        __threadfence();
        const unsigned int t = atomicAdd(ticket, 1u);
        amLast = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!amLast) return false;
    __threadfence();
    double acc[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) acc[r] = 0.0;
    // each thread adds the partials i, i + NT, i + 2 NT, ... in that order;
    // U of them are loaded before any is added, so their L2 round trips
    // overlap (the order of the additions is unchanged)
    constexpr int U = NR >= 8 ? 1 : 8 / NR;
    const int G = (int)gridDim.x;
    int i = threadIdx.x;
    for (; i + (U - 1) * NT < G; i += U * NT)
    {
        double t[NR][U];
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int r = 0; r < NR; ++r) t[r][u] = __ldcg(part + r * G + i + u * NT);
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int r = 0; r < NR; ++r) acc[r] += t[r][u];
    }
    for (; i < G; i += NT)
    {
#pragma unroll
        for (int r = 0; r < NR; ++r) acc[r] += __ldcg(part + r * G + i);
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

// Grid-wide max (same protocol as grid_sum).
__device__ __forceinline__ bool grid_max(double& v, double* part,
                                         unsigned int* ticket)
{
    __shared__ double sh[NT / 32];
    __shared__ bool amLast;
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    v = warp_max(v);
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    if (threadIdx.x == 0)
    {
        double m = sh[0];
        for (int w = 1; w < NT / 32; ++w) m = fmax(m, sh[w]);
        part[blockIdx.x] = m;
        __threadfence();
        const unsigned int t = atomicAdd(ticket, 1u);
        amLast = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!amLast) return false;
    __threadfence();
    double m = -INFINITY;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += NT) m = fmax(m, __ldcg(part + i));
    m = warp_max(m);
    __syncthreads();
    if (lane == 0) sh[wid] = m;
    __syncthreads();
    if (threadIdx.x == 0)
    {
        double t = sh[0];
        for (int w = 1; w < NT / 32; ++w) t = fmax(t, sh[w]);
        v = t;
        *ticket = 0u;
    }
    return true;
}

// Bounded grid barrier of a cooperative (all blocks co-resident) launch:
// generation counter in global memory, the last block to arrive resets the
// count and bumps the generation.  A block that has polled `polls` times
// gives up: it sets the error word and the barrier returns false in every
// block that sees it, so the kernel ends instead of waiting (the host then
// reports CF_ERR_DEVICE_TIMEOUT).
struct GridBar
{
    unsigned int* count;
    unsigned int* gen;
    int* err;
    unsigned long long polls;
};

__device__ __forceinline__ bool grid_barrier(const GridBar& b)
{
    __syncthreads();
    if (threadIdx.x == 0)
    {
        volatile unsigned int* vgen = b.gen;
        const unsigned int g = *vgen;
        __threadfence();
        if (atomicAdd(b.count, 1u) == gridDim.x - 1)
        {
            *b.count = 0u;
            __threadfence();
            atomicAdd(b.gen, 1u);
        }
        else
        {
            unsigned long long spins = 0;
            while (*vgen == g)
            {
                if (++spins > b.polls)
                {
                    atomicExch(b.err, 1);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return *(volatile int*)b.err == 0;
}

__device__ __forceinline__ int free_buffer(int a, int b)
{
    for (int i = 0; i < 3; ++i)
        if (i != a && i != b) return i;
    return 0;
}

__device__ __forceinline__ bool is_nbr(int c) { return c < -1; }
__device__ __forceinline__ bool is_own(int c) { return c >= 0; }
__device__ __forceinline__ int col_index(int c) { return c & 0x7fffffff; }

// One FP32 row of A x: acc (= diag*x_row) plus the entries in stored order
// (owner side, then neighbour side), as ldu_spmv (metalFoamKernels.metal:131-147).
// PAIRED = W (PAIR_MIN_W..PAIR_MAX_W) reads the paired copy of the compact
// stream (A.pcol16/A.pval) of a layout whose slices all have width W;
// PAIRED = 0 the column-major streams.  A kernel is compiled for one of
// them, so neither pays registers or branches for the other.
template <int MAXW, int PAIRED = 0, class XF>
__device__ __forceinline__ float row_f32(const DevSell& A, int row, float acc,
                                         XF xf)
{
    if constexpr (PAIRED != 0)
    {
        // paired order: one short2 and one float2 load per two entries (the
        // last entry of an odd width alone); same entries, summed in the
        // same order (offsets fit 32 bits: the layout is refused beyond
        // 2^31 entries)
        constexpr int W = PAIRED;
        constexpr int EVEN = W & ~1;
        const int sb = (row >> 5) * SLICE * W;
        const int lane = row & 31;
        short o[W];
        float v[W];
#pragma unroll
        for (int g = 0; g < EVEN / 2; ++g)
        {
            const int e = sb + 64 * g + 2 * lane;
            const short2 oo = __ldcs(reinterpret_cast<const short2*>(A.pcol16 + e));
            const float2 vv = __ldcs(reinterpret_cast<const float2*>(A.pval + e));
            o[2 * g] = oo.x;
            o[2 * g + 1] = oo.y;
            v[2 * g] = vv.x;
            v[2 * g + 1] = vv.y;
        }
        if constexpr (W != EVEN)
        {
            const int e = sb + 32 * EVEN + lane;
            o[W - 1] = __ldcs(A.pcol16 + e);
            v[W - 1] = __ldcs(A.pval + e);
        }
        float x[W];
#pragma unroll
        for (int k = 0; k < W; ++k) x[k] = (o[k] != COL16_PAD) ? xf(row + o[k]) : 0.0f;
#pragma unroll
        for (int k = 0; k < W; ++k)
            if (o[k] != COL16_PAD) acc = __fadd_rn(acc, __fmul_rn(v[k], x[k]));
        return acc;
    }
    else
    {
    const int s = row >> 5;
    const int b0 = A.ellW ? s * SLICE * A.ellW : __ldg(A.sliceOff + s);
    const int w = A.ellW ? A.ellW : (__ldg(A.sliceOff + s + 1) - b0) >> 5;
    const int base = b0 + (row & 31);
    if (A.col16)
    {
        // compact index stream: same columns, same order, half the bytes
        if (w <= MAXW)
        {
            short o[MAXW];
            float v[MAXW];
#pragma unroll
            for (int k = 0; k < MAXW; ++k)
            {
                if (k < w)
                {
                    o[k] = __ldcs(A.col16 + base + SLICE * k);
                    v[k] = __ldcs(A.val + base + SLICE * k);
                }
                else
                {
                    o[k] = COL16_PAD;
                    v[k] = 0.0f;
                }
            }
            float x[MAXW];
#pragma unroll
            for (int k = 0; k < MAXW; ++k) x[k] = (o[k] != COL16_PAD) ? xf(row + o[k]) : 0.0f;
#pragma unroll
            for (int k = 0; k < MAXW; ++k)
                if (o[k] != COL16_PAD) acc = __fadd_rn(acc, __fmul_rn(v[k], x[k]));
        }
        else
        {
            for (int k = 0; k < w; ++k)
            {
                const short o = __ldcs(A.col16 + base + SLICE * k);
                if (o != COL16_PAD)
                    acc = __fadd_rn(acc, __fmul_rn(__ldcs(A.val + base + SLICE * k), xf(row + o)));
            }
        }
        return acc;
    }
    if (w <= MAXW)
    {
        int c[MAXW];
        float v[MAXW];
#pragma unroll
        for (int k = 0; k < MAXW; ++k)
        {
            if (k < w)
            {
                c[k] = __ldcs(A.col + base + SLICE * k);
                v[k] = __ldcs(A.val + base + SLICE * k);
            }
            else
            {
                c[k] = -1;
                v[k] = 0.0f;
            }
        }
        float x[MAXW];
#pragma unroll
        for (int k = 0; k < MAXW; ++k) x[k] = (c[k] != -1) ? xf(col_index(c[k])) : 0.0f;
#pragma unroll
        for (int k = 0; k < MAXW; ++k)
            if (c[k] != -1) acc = __fadd_rn(acc, __fmul_rn(v[k], x[k]));
    }
    else
    {
        for (int k = 0; k < w; ++k)
        {
            const int c = __ldcs(A.col + base + SLICE * k);
            if (c != -1)
                acc = __fadd_rn(acc, __fmul_rn(__ldcs(A.val + base + SLICE * k),
                                               xf(col_index(c))));
        }
    }
    return acc;
    }
}

// One FP64 row: acc (= diag*x_row) plus neighbour-side entries, then
// owner-side entries -- lduMatrix::Amul's per-row order.  `vals` is val64
// (A) or the transposed values (A^T).
template <int MAXW, class XF>
__device__ __forceinline__ double row_f64(const DevSell& A, const double* vals,
                                          int row, double acc, XF xf)
{
    const int s = row >> 5;
    const int b0 = A.ellW ? s * SLICE * A.ellW : __ldg(A.sliceOff + s);
    const int w = A.ellW ? A.ellW : (__ldg(A.sliceOff + s + 1) - b0) >> 5;
    const int base = b0 + (row & 31);
    if (w <= MAXW)
    {
        int c[MAXW];
        double v[MAXW];
        double x[MAXW];
#pragma unroll
        for (int k = 0; k < MAXW; ++k)
        {
            if (k < w)
            {
                c[k] = __ldcs(A.col + base + SLICE * k);
                v[k] = __ldcs(vals + base + SLICE * k);
            }
            else
            {
                c[k] = -1;
                v[k] = 0.0;
            }
        }
#pragma unroll
        for (int k = 0; k < MAXW; ++k) x[k] = (c[k] != -1) ? xf(col_index(c[k])) : 0.0;
#pragma unroll
        for (int k = 0; k < MAXW; ++k)
            if (is_nbr(c[k])) acc = __dadd_rn(acc, __dmul_rn(v[k], x[k]));
#pragma unroll
        for (int k = 0; k < MAXW; ++k)
            if (is_own(c[k])) acc = __dadd_rn(acc, __dmul_rn(v[k], x[k]));
    }
    else
    {
        for (int k = 0; k < w; ++k)
        {
            const int c = __ldcs(A.col + base + SLICE * k);
            if (is_nbr(c))
                acc = __dadd_rn(acc, __dmul_rn(__ldcs(vals + base + SLICE * k), xf(col_index(c))));
        }
        for (int k = 0; k < w; ++k)
        {
            const int c = __ldcs(A.col + base + SLICE * k);
            if (is_own(c))
                acc = __dadd_rn(acc, __dmul_rn(__ldcs(vals + base + SLICE * k), xf(col_index(c))));
        }
    }
    return acc;
}

#define CF_ROWS(row, n) \
    for (int row = blockIdx.x * NT + threadIdx.x; row < (n); row += gridDim.x * NT)

// ------------------------------------------------------ coefficient staging

// val32/val64 from the face arrays (setCoeffs, metalFoamBackend.C:533-555):
// owner-side entries take upper[f], neighbour-side entries lower[f] (or
// upper[f] when the FP32 matrix is staged symmetric, as the reference does
// for PCG, metalFoamSolver.C:216-218).  valT64 holds A^T's values.
static __global__ void k_stage_vals(long long nnzp, const int* __restrict__ col,
                             const int* __restrict__ eface,
                             const double* __restrict__ upper,
                             const double* __restrict__ lower, int sym32,
                             float* __restrict__ val32, double* __restrict__ val64,
                             double* __restrict__ valT64)
{
    for (long long e = (long long)blockIdx.x * NT + threadIdx.x; e < nnzp;
         e += (long long)gridDim.x * NT)
    {
        const int f = eface[e];
        if (f < 0)
        {
            val32[e] = 0.0f;
            val64[e] = 0.0;
            valT64[e] = 0.0;
            continue;
        }
        const bool nbr = is_nbr(col[e]);
        const double u = upper[f];
        const double l = lower[f];
        const double a = nbr ? l : u;
        val64[e] = a;
        valT64[e] = nbr ? u : l;
        val32[e] = (float)((sym32 && nbr) ? u : a);
    }
}

// val32 in the paired order of a uniform-width-W layout (see pair_index)
static __global__ void k_pair_vals(long long nnzp, int W, const float* __restrict__ val32,
                                   float* __restrict__ pval)
{
    const long long sw = (long long)SLICE * W;
    for (long long e = (long long)blockIdx.x * NT + threadIdx.x; e < nnzp;
         e += (long long)gridDim.x * NT)
    {
        const long long s = e / sw;
        const int rem = (int)(e - s * sw);
        pval[pair_index(s * sw, W, rem / SLICE, rem % SLICE)] = val32[e];
    }
}

static __global__ void k_gather_f64(int n, const int* __restrict__ perm,
                             const double* __restrict__ src, double* __restrict__ dst)
{
    CF_ROWS(row, n) dst[row] = src[perm[row]];
}

static __global__ void k_scatter_f64(int n, const int* __restrict__ perm,
                              const double* __restrict__ src, double* __restrict__ dst)
{
    CF_ROWS(row, n) dst[perm[row]] = src[row];
}

static __global__ void k_gather_f32(int n, const int* __restrict__ perm,
                             const float* __restrict__ src, float* __restrict__ dst)
{
    CF_ROWS(row, n) dst[row] = src[perm[row]];
}

static __global__ void k_scatter_f32(int n, const int* __restrict__ perm,
                              const float* __restrict__ src, float* __restrict__ dst)
{
    CF_ROWS(row, n) dst[perm[row]] = src[row];
}

// u = A 1 (sumA), the deflation census of metalFoamSolver.C:182-188 and the
// sign test of the deflated diagonal (metalFoamSolver.C:199-207).
template <int MAXW>
static __global__ void __launch_bounds__(NT) k_sumA(DevSell A, const double* __restrict__ diag64,
                                             double* __restrict__ u, DriverState* drv,
                                             double* part)
{
    double acc[2] = {0.0, 0.0};
    CF_ROWS(row, A.n)
    {
        const double d = diag64[row];
        const double s = row_f64<MAXW>(A, A.val64, row, d, [](int) { return 1.0; });
        u[row] = s;
        if (fabs(s) > 1e-8 * fabs(d)) acc[0] += 1.0;
        const double d0 = __dsub_rn(d, s);
        if (__dmul_rn(d0, d) <= VSMALL * fabs(d0)) acc[1] += 1.0;
    }
    if (grid_sum<2>(acc, part, &drv->ticket) && threadIdx.x == 0)
    {
        drv->nPinned = (long long)acc[0];
        drv->signflip = acc[1] > 0.0;
    }
}

// FP32 diagonal and reciprocal of the chosen diagonal (deflated: diag - u).
static __global__ void k_stage_diag32(int n, const double* __restrict__ diag64,
                               const double* __restrict__ u, int deflate,
                               float* __restrict__ diag32, float* __restrict__ rD32)
{
    CF_ROWS(row, n)
    {
        const double dp = deflate ? __dsub_rn(diag64[row], u[row]) : diag64[row];
        diag32[row] = (float)dp;
        rD32[row] = (float)(1.0 / dp);
    }
}

// Gershgorin bound of D^-1 A (metalFoamSolver.C:229-249):
// max_i (1 + sum_{faces of i} |upper_f| / |diagPtr_i|), summed per row in the
// face-loop order; then the Chebyshev constants.
template <int MAXW>
static __global__ void __launch_bounds__(NT) k_gershgorin(DevSell A, const int* __restrict__ eface,
                                                   const double* __restrict__ upper,
                                                   const double* __restrict__ diag64,
                                                   const double* __restrict__ u, int deflate,
                                                   int order, double ratio,
                                                   float* __restrict__ chebC,
                                                   DriverState* drv, double* part)
{
    double m = 0.0;
    CF_ROWS(row, A.n)
    {
        const int s = row >> 5;
        const int b0 = A.sliceOff[s];
        const int w = (A.sliceOff[s + 1] - b0) >> 5;
        const int base = b0 + (row & 31);
        double so = 0.0;
        for (int k = 0; k < w; ++k)
        {
            const int c = A.col[base + SLICE * k];
            if (is_nbr(c)) so = __dadd_rn(so, fabs(upper[eface[base + SLICE * k]]));
        }
        for (int k = 0; k < w; ++k)
        {
            const int c = A.col[base + SLICE * k];
            if (is_own(c)) so = __dadd_rn(so, fabs(upper[eface[base + SLICE * k]]));
        }
        const double dp = deflate ? __dsub_rn(diag64[row], u[row]) : diag64[row];
        const double g = __dadd_rn(1.0, so / fabs(dp));
        m = fmax(m, g);
    }
    if (grid_max(m, part, &drv->ticket) && threadIdx.x == 0)
    {
        drv->chebBeta = m;
        cheb_constants(order, m, ratio, chebC);
    }
}

// ------------------------------------------------------------ FP64 driver

static __global__ void __launch_bounds__(NT) k_mean_f64(int n, const double* __restrict__ x,
                                                 double* out, unsigned int* ticket,
                                                 double* part)
{
    double acc[1] = {0.0};
    CF_ROWS(row, n) acc[0] += x[row];
    if (grid_sum<1>(acc, part, ticket) && threadIdx.x == 0) *out = acc[0] / (double)n;
}

// mean of the correction selected by the last inner solve (FP32 values)
static __global__ void __launch_bounds__(NT) k_mean_delta(int n, const float* __restrict__ D,
                                                   const InnerState* st, double* out,
                                                   unsigned int* ticket, double* part)
{
    const float* d = D + (size_t)st->sel * n;
    double acc[1] = {0.0};
    CF_ROWS(row, n) acc[0] += (double)d[row];
    if (grid_sum<1>(acc, part, ticket) && threadIdx.x == 0) *out = acc[0] / (double)n;
}

// wA = A psi; r = b - wA; normFactor (L1_SCALED, xRef = mean psi) and the
// initial residual (metalFoamSolver.C:109-128).
template <int MAXW>
static __global__ void __launch_bounds__(NT) k_residual0(DevSell A, const double* __restrict__ diag64,
                                                  const double* __restrict__ psi,
                                                  const double* __restrict__ b,
                                                  const double* __restrict__ u,
                                                  double* __restrict__ r64, DriverState* drv,
                                                  double* part)
{
    const double xbar = drv->xbar;
    double acc[2] = {0.0, 0.0};
    CF_ROWS(row, A.n)
    {
        const double wa = row_f64<MAXW>(A, A.val64, row, __dmul_rn(diag64[row], psi[row]),
                                        [&](int c) { return __ldg(psi + c); });
        const double bb = b[row];
        const double rr = __dsub_rn(bb, wa);
        r64[row] = rr;
        const double pA = __dmul_rn(u[row], xbar);
        acc[0] += __dadd_rn(fabs(__dsub_rn(wa, pA)), fabs(__dsub_rn(bb, pA)));
        acc[1] += fabs(rr);
    }
    if (grid_sum<2>(acc, part, &drv->ticket) && threadIdx.x == 0)
    {
        drv->normFactor = acc[0] + 1e-20;
        drv->initRes = acc[1] / drv->normFactor;
        drv->finalRes = drv->initRes;
    }
}

// r = b - A psi (metalFoamSolver.C:333-340); without deflation also the
// normalised L1 residual, with deflation the u.r and u.u sums of the
// constant-mode shift (metalFoamSolver.C:344-351).
template <int MAXW>
static __global__ void __launch_bounds__(NT) k_residual(DevSell A, const double* __restrict__ diag64,
                                                 const double* __restrict__ psi,
                                                 const double* __restrict__ b,
                                                 const double* __restrict__ u,
                                                 double* __restrict__ r64, int deflate,
                                                 DriverState* drv, double* part)
{
    double acc[2] = {0.0, 0.0};
    CF_ROWS(row, A.n)
    {
        const double wa = row_f64<MAXW>(A, A.val64, row, __dmul_rn(diag64[row], psi[row]),
                                        [&](int c) { return __ldg(psi + c); });
        const double rr = __dsub_rn(b[row], wa);
        r64[row] = rr;
        if (deflate)
        {
            const double uu = u[row];
            acc[0] += uu * rr;
            acc[1] += uu * uu;
        }
        else
        {
            acc[0] += fabs(rr);
        }
    }
    if (grid_sum<2>(acc, part, &drv->ticket) && threadIdx.x == 0)
    {
        if (deflate)
        {
            drv->ur = acc[0];
            drv->uu = acc[1];
        }
        else
        {
            drv->finalRes = acc[0] / drv->normFactor;
        }
    }
}

// psi += c, r -= c u with c = (u.r)/(u.u) when u.u > VSMALL
// (metalFoamSolver.C:352-361), then the normalised L1 residual.
static __global__ void __launch_bounds__(NT) k_cshift(int n, double* __restrict__ psi,
                                               double* __restrict__ r64,
                                               const double* __restrict__ u,
                                               DriverState* drv, double* part)
{
    const double ur = drv->ur;
    const double uu = drv->uu;
    const bool apply = uu > VSMALL;
    const double c = apply ? ur / uu : 0.0;
    double acc[1] = {0.0};
    CF_ROWS(row, n)
    {
        double rr = r64[row];
        if (apply)
        {
            psi[row] = __dadd_rn(psi[row], c);
            rr = __dsub_rn(rr, __dmul_rn(c, u[row]));
            r64[row] = rr;
        }
        acc[0] += fabs(rr);
    }
    if (grid_sum<1>(acc, part, &drv->ticket) && threadIdx.x == 0)
        drv->finalRes = acc[0] / drv->normFactor;
}

// psi += double(delta) - mean(delta) (metalFoamSolver.C:318-330)
static __global__ void k_psi_update(int n, double* __restrict__ psi, const float* __restrict__ D,
                             const InnerState* st, const double* dmean)
{
    const float* d = D + (size_t)st->sel * n;
    const double m = dmean ? *dmean : 0.0;
    CF_ROWS(row, n) psi[row] = __dadd_rn(psi[row], __dsub_rn((double)d[row], m));
}

static __global__ void __launch_bounds__(NT) k_l2(int n, const double* __restrict__ r64,
                                           const double* __restrict__ b, DriverState* drv,
                                           double* part)
{
    double acc[2] = {0.0, 0.0};
    CF_ROWS(row, n)
    {
        acc[0] += r64[row] * r64[row];
        acc[1] += b[row] * b[row];
    }
    if (grid_sum<2>(acc, part, &drv->ticket) && threadIdx.x == 0)
    {
        drv->l2r = sqrt(acc[0]);
        drv->l2b = sqrt(acc[1]);
    }
}

// FP64 y = A x (or A^T x with valT64), Amul order.
template <int MAXW>
static __global__ void __launch_bounds__(NT) k_amul64(DevSell A, const double* __restrict__ vals,
                                               const double* __restrict__ diag64,
                                               const double* __restrict__ x,
                                               double* __restrict__ y)
{
    CF_ROWS(row, A.n)
    y[row] = row_f64<MAXW>(A, vals, row, __dmul_rn(diag64[row], x[row]),
                           [&](int c) { return __ldg(x + c); });
}

// ------------------------------------------------------------ inner solves

// rows whose loads k_pcg_update issues together per thread (2 keeps it at
// 32 registers, the occupancy and grid of one row at a time)
constexpr int PCG_UPDATE_ROWS = 2;

struct PcgBufs
{
    float* rA;          // FP32 residual
    float* W0;          // Chebyshev w0 (= z0) or Jacobi wA = rD rA
    float* W1;          // Chebyshev w for steps >= 1
    float* Z0;          // Chebyshev z ping-pong
    float* Z1;
    float* P;           // [2n] search direction ping-pong (by iteration parity)
    float* Q;           // A p
    float* D;           // [3n] corrections (cur / best / next)
    const float* diag;  // FP32 diag (possibly deflated)
    const float* rD;    // FP32 1/diag
    const float* chebC; // Chebyshev constants
    const double* r64;  // inner right-hand side (FP64)
    int n;
};

static __global__ void k_inner_setup(InnerState* st, double target, int maxIter, int ips,
                                     int stagLimit = STAG_LIMIT)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    st->stagLimit = stagLimit > 0 ? stagLimit : STAG_LIMIT;
    st->wArA = st->wArAold = st->wApA = st->alpha = st->beta = st->res = 0.0;
    st->rA0rA = st->rA0rAold = st->rA0AyA = st->omega = st->tAtA = st->tAsA = st->resS = 0.0;
    st->bestRes = 1.0e300;
    st->target = target;
    st->finalResSum = 0.0;
    st->it = 0;
    st->maxIter = maxIter;
    st->ips = ips < 1 ? 1 : ips;
    st->lastSync = 0;
    st->noProgress = 0;
    st->cur = 0;
    st->best = 0;
    st->nxt = 1;
    st->converged = st->singular = st->stagnated = st->done = st->early = 0;
    st->sel = 0;
    st->ticket = 0u;
}

// Start of the inner PCG (metalFoamBackend.C:593-597 plus the first
// preconditioner apply): rA = float(r - mean), delta = p = 0, then
// cheb_init (w0 = c1 rD rA) or pcg_precond_dot (wA = rA rD and wA.rA,
// reduce_scalars mode 0 with firstIter: beta = 0).
template <bool CHEB>
static __global__ void __launch_bounds__(NT) k_pcg_init(PcgBufs B, const double* mean,
                                                 InnerState* st, double* part)
{
    const int n = B.n;
    const double m = mean ? *mean : 0.0;
    const float c1 = CHEB ? B.chebC[0] : 0.0f;
    double acc[1] = {0.0};
    CF_ROWS(row, n)
    {
        const float ra = (float)(B.r64[row] - m);
        B.rA[row] = ra;
        B.D[row] = 0.0f;
        B.P[row] = 0.0f;
        B.P[n + row] = 0.0f;
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
        if (grid_sum<1>(acc, part, &st->ticket) && threadIdx.x == 0)
        {
            st->wArAold = st->wArA;
            st->wArA = acc[0];
            st->beta = 0.0;
        }
    }
}

// Chebyshev step j (cheb_step after ldu_spmv, metalFoamKernels.metal:113-194,
// encoded per step at metalFoamBackend.C:365-384) fused into one pass:
//   v = A z_{j-1};  w = c2 w + c3 rD (r - v);  z_j = z_{j-1} + w.
// On the last step the z.r dot and reduce_scalars mode 0 (wArA, beta) follow.
// The last step (with the z.r sum) runs on its occupancy grid, the other
// steps one row per thread (rows_grid).
template <bool LAST, int MAXW, int PAIRED = 0>
static __global__ void __launch_bounds__(NT) k_cheb_step(DevSell A, PcgBufs B, const float* zin,
                                                  const float* win, float* wout, float* zout,
                                                  int j, InnerState* st, double* part)
{
    if (st->done) return;
    const float c2 = B.chebC[2 * j - 1];
    const float c3 = B.chebC[2 * j];
    double acc[1] = {0.0};
    CF_ROWS(row, A.n)
    {
        const float zr = zin[row];
        const float v = row_f32<MAXW, PAIRED>(A, row, __fmul_rn(B.diag[row], zr),
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
        if (grid_sum<1>(acc, part, &st->ticket) && threadIdx.x == 0)
        {
            st->wArAold = st->wArA;
            st->wArA = acc[0];
            st->beta = (st->it == 0) ? 0.0 : st->wArA / st->wArAold;
        }
    }
}

// pcg_update_p fused into ldu_spmv_dotw (metalFoamKernels.metal:64-109,237-247):
// p_new = wA + beta p_old is formed on the fly for every gathered column, so
// p never needs its own pass; writes p_new, q = A p_new; p.q -> alpha
// (reduce_scalars mode 1).
template <int MAXW, int PAIRED = 0>
static __global__ void __launch_bounds__(NT) k_pcg_p_spmv(DevSell A, PcgBufs B, const float* wA,
                                                   InnerState* st, double* part)
{
    if (st->done) return;
    const int n = A.n;
    const int par = st->it & 1;
    const float* __restrict__ Pold = B.P + (size_t)(par ^ 1) * n;
    float* __restrict__ Pn = B.P + (size_t)par * n;
    const float beta = (float)st->beta;
    auto pf = [&](int c) { return __fadd_rn(__ldg(wA + c), __fmul_rn(beta, __ldg(Pold + c))); };
    double acc[1] = {0.0};
    CF_ROWS(row, n)
    {
        const float pr = pf(row);
        const float y = row_f32<MAXW, PAIRED>(A, row, __fmul_rn(B.diag[row], pr), pf);
        Pn[row] = pr;
        B.Q[row] = y;
        acc[0] += (double)pr * (double)y;
    }
    if (grid_sum<1>(acc, part, &st->ticket) && threadIdx.x == 0)
    {
        st->wApA = acc[0];
        st->alpha = st->wArA / st->wApA;
    }
}

// End-of-iteration bookkeeping of metalFoamBackend::pcg (.C:676-715) on the
// device: breakdown, minimum-residual iterate, convergence, stagnation, at
// every batch boundary of iterationsPerSync.
// (S = InnerState, or volatile InnerState inside a persistent kernel, whose
// state must not be served from a stale L1 line)
template <class S>
__device__ __forceinline__ void inner_sync_point(S* st, bool checkWApA)
{
    const int it = st->it;
    const bool sync = (it - st->lastSync >= st->ips) || (it >= st->maxIter);
    if (sync)
    {
        const int batch = it - st->lastSync;
        st->lastSync = it;
        const double res = st->res;
        st->finalResSum = res;
        const bool bad = !isfinite(res) || (checkWApA ? !isfinite(st->wApA) : !isfinite(st->omega));
        if (bad)
        {
            st->singular = 1;
            st->done = 1;
        }
        else
        {
            if (res < st->bestRes)
            {
                st->bestRes = res;
                st->best = st->cur;
                st->noProgress = 0;
            }
            else
            {
                st->noProgress += batch;
            }
            if (res <= st->target)
            {
                st->converged = 1;
                st->done = 1;
            }
            else if (st->noProgress >= st->stagLimit)
            {
                st->stagnated = 1;
                st->done = 1;
            }
        }
    }
    if (it >= st->maxIter) st->done = 1;
    st->nxt = free_buffer(st->cur, st->best);
}

// pcg_update_sol_res (metalFoamKernels.metal:251-276) + the next iteration's
// preconditioner start: delta_next = delta + alpha p; rA -= alpha q; sum|rA|;
// Chebyshev: w0 = c1 rD rA; Jacobi: wA = rA rD and wA.rA (beta).
// Each thread takes its rows row, row + stride, ... in that order (the fold
// order of the sums); U of them have their five loads issued before the
// first is updated, so a thread keeps 5 U loads in flight instead of 5.
template <bool CHEB, int U = PCG_UPDATE_ROWS>
static __global__ void __launch_bounds__(NT) k_pcg_update(PcgBufs B, InnerState* st, double* part,
                                                   cudaGraphConditionalHandle h, int useCond)
{
    if (st->done) return;
    const int n = B.n;
    const int par = st->it & 1;
    const float* __restrict__ P = B.P + (size_t)par * n;
    const float* __restrict__ D = B.D + (size_t)st->cur * n;
    float* __restrict__ Dn = B.D + (size_t)st->nxt * n;
    const float alpha = (float)st->alpha;
    const float c1 = CHEB ? B.chebC[0] : 0.0f;
    double acc[2] = {0.0, 0.0};
    auto one = [&](int row, float d, float p, float r, float q, float rd) {
        Dn[row] = __fadd_rn(d, __fmul_rn(alpha, p));
        const float rn = __fsub_rn(r, __fmul_rn(alpha, q));
        B.rA[row] = rn;
        acc[0] += (double)fabsf(rn);
        if (CHEB)
        {
            B.W0[row] = __fmul_rn(__fmul_rn(c1, rd), rn);
        }
        else
        {
            const float wa = __fmul_rn(rn, rd);
            B.W0[row] = wa;
            acc[1] += (double)wa * (double)rn;
        }
    };
    const int stride = gridDim.x * NT;
    int row = blockIdx.x * NT + threadIdx.x;
    for (; row + (U - 1) * stride < n; row += U * stride)
    {
        float d[U], p[U], r[U], q[U], rd[U];
#pragma unroll
        for (int u = 0; u < U; ++u)
        {
            const int i = row + u * stride;
            d[u] = D[i];
            p[u] = P[i];
            r[u] = B.rA[i];
            q[u] = B.Q[i];
            rd[u] = B.rD[i];
        }
#pragma unroll
        for (int u = 0; u < U; ++u) one(row + u * stride, d[u], p[u], r[u], q[u], rd[u]);
    }
    for (; row < n; row += stride) one(row, D[row], P[row], B.rA[row], B.Q[row], B.rD[row]);
    if (grid_sum<2>(acc, part, &st->ticket) && threadIdx.x == 0)
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
        if (useCond) cudaGraphSetConditional(h, st->done ? 0u : 1u);
    }
}

// Return the best iterate seen (metalFoamBackend.C:718-727); BiCGStab's
// early exit returns its last iterate (.C:841-865).
static __global__ void k_inner_final(InnerState* st)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (st->early)
    {
        st->sel = st->cur;
    }
    else if (st->bestRes < st->finalResSum)
    {
        st->sel = st->best;
        st->finalResSum = st->bestRes;
    }
    else
    {
        st->sel = st->cur;
    }
}

struct BicgBufs
{
    float* rA;
    float* rA0;
    float* P;           // [2n] search direction ping-pong (by iteration parity)
    float* yA;
    float* AyA;         // [2n] A yA ping-pong (by iteration parity)
    float* sA;
    float* zA;
    float* tA;
    float* D;           // [3n]
    const float* diag;
    const float* rD;
    const double* r64;
    int n;
};

// Start of the inner BiCGStab (metalFoamBackend.C:761-770): rA, rA0 = rA,
// delta = p = AyA = 0 (both parities: iteration 0 reads the odd ones as
// "previous"); then rA0.rA and reduce_scalars mode 3 (firstIter).
static __global__ void __launch_bounds__(NT) k_bicg_init(BicgBufs B, const double* mean,
                                                  InnerState* st, double* part)
{
    const int n = B.n;
    const double m = mean ? *mean : 0.0;
    double acc[1] = {0.0};
    CF_ROWS(row, n)
    {
        const float ra = (float)(B.r64[row] - m);
        B.rA[row] = ra;
        B.rA0[row] = ra;
        B.D[row] = 0.0f;
        B.P[row] = 0.0f;
        B.P[n + row] = 0.0f;
        B.AyA[row] = 0.0f;
        B.AyA[n + row] = 0.0f;
        acc[0] += (double)ra * (double)ra;
    }
    if (grid_sum<1>(acc, part, &st->ticket) && threadIdx.x == 0)
    {
        st->rA0rAold = st->rA0rA;
        st->rA0rA = acc[0];
        st->beta = 0.0;
    }
}

// bicg_update_p + emul (metalFoamKernels.metal:198-208,372-386) fused into
// the SpMV ldu_spmv_dotw + reduce_scalars mode 4: p = rA + beta (p_old -
// omega AyA_old) and yA = rD p are formed on the fly for every gathered
// column (the previous iteration's p and AyA sit in the other parity), so
// they need no pass of their own; writes p, yA, AyA = A yA for the own row;
// rA0.AyA -> alpha.
template <int MAXW, int PAIRED = 0>
static __global__ void __launch_bounds__(NT) k_bicg_ab(DevSell A, BicgBufs B, InnerState* st,
                                                double* part)
{
    if (st->done) return;
    const int n = A.n;
    const int par = st->it & 1;
    const float* __restrict__ Pold = B.P + (size_t)(par ^ 1) * n;
    const float* __restrict__ Aold = B.AyA + (size_t)(par ^ 1) * n;
    float* __restrict__ Pn = B.P + (size_t)par * n;
    float* __restrict__ An = B.AyA + (size_t)par * n;
    const float beta = (float)st->beta;
    const float omega = (float)st->omega;
    auto pf = [&](int c) {
        return __fadd_rn(__ldg(B.rA + c),
                         __fmul_rn(beta, __fsub_rn(__ldg(Pold + c), __fmul_rn(omega, __ldg(Aold + c)))));
    };
    auto yf = [&](int c) { return __fmul_rn(__ldg(B.rD + c), pf(c)); };
    double acc[1] = {0.0};
    CF_ROWS(row, n)
    {
        const float p = pf(row);
        const float y = __fmul_rn(B.rD[row], p);
        Pn[row] = p;
        B.yA[row] = y;
        const float v = row_f32<MAXW, PAIRED>(A, row, __fmul_rn(B.diag[row], y), yf);
        An[row] = v;
        acc[0] += (double)B.rA0[row] * (double)v;
    }
    if (grid_sum<1>(acc, part, &st->ticket) && threadIdx.x == 0)
    {
        st->rA0AyA = acc[0];
        st->alpha = st->rA0rA / st->rA0AyA;
    }
}

// bicg_s_res + emul (metalFoamKernels.metal:390-412) fused into the second
// SpMV (reduce_scalars mode 5): s = rA - alpha AyA and zA = rD s are formed
// on the fly for every gathered column; writes sA, zA, tA = A zA for the own
// row; sum|s|, s.tA and tA.tA in one reduction.  The finaliser applies the
// host checks of metalFoamBackend.C:829-866 first -- breakdown on rA0rA /
// alpha / sum|s|, the |s| early exit -- and only then omega = s.tA / tA.tA.
template <int MAXW, int PAIRED = 0>
static __global__ void __launch_bounds__(NT) k_bicg_cd(DevSell A, BicgBufs B, InnerState* st,
                                                double* part, cudaGraphConditionalHandle h,
                                                int useCond)
{
    if (st->done) return;
    const int n = A.n;
    const int par = st->it & 1;
    const float* __restrict__ An = B.AyA + (size_t)par * n;
    const float alpha = (float)st->alpha;
    auto zf = [&](int c) {
        return __fmul_rn(__ldg(B.rD + c), __fsub_rn(__ldg(B.rA + c), __fmul_rn(alpha, __ldg(An + c))));
    };
    double acc[3] = {0.0, 0.0, 0.0};
    CF_ROWS(row, n)
    {
        const float sv = __fsub_rn(B.rA[row], __fmul_rn(alpha, An[row]));
        const float z = __fmul_rn(B.rD[row], sv);
        B.sA[row] = sv;
        B.zA[row] = z;
        acc[0] += (double)fabsf(sv);
        const float t = row_f32<MAXW, PAIRED>(A, row, __fmul_rn(B.diag[row], z), zf);
        B.tA[row] = t;
        acc[1] += (double)sv * (double)t;
        acc[2] += (double)t * (double)t;
    }
    if (grid_sum<3>(acc, part, &st->ticket) && threadIdx.x == 0)
    {
        st->resS = acc[0];
        if (!isfinite(st->rA0rA) || !isfinite(st->alpha) || !isfinite(st->resS))
        {
            st->singular = 1;
            st->done = 1;
        }
        else if (st->resS <= st->target)
        {
            st->early = 1;
            st->done = 1;
        }
        else
        {
            st->tAsA = acc[1];
            st->tAtA = acc[2];
            st->omega = st->tAsA / st->tAtA;
        }
        if (useCond && st->done) cudaGraphSetConditional(h, 0u);
    }
}

// bicg_update_sol_res (metalFoamKernels.metal:430-458) + the end-of-iteration
// checks (metalFoamBackend.C:908-943) + the next iteration's rA0.rA and
// beta (reduce_scalars mode 3).  On the |s| early exit instead delta +=
// alpha yA (bicg_early_update) and the solve ends.
static __global__ void __launch_bounds__(NT) k_bicg_e(BicgBufs B, InnerState* st, double* part,
                                               cudaGraphConditionalHandle h, int useCond)
{
    const bool early = st->early;
    if (st->done && !early) return;
    const int n = B.n;
    const float alpha = (float)st->alpha;
    const float* __restrict__ D = B.D + (size_t)st->cur * n;
    float* __restrict__ Dn = B.D + (size_t)st->nxt * n;
    double acc[2] = {0.0, 0.0};
    if (early)
    {
        if (st->converged) return;   // already applied
        CF_ROWS(row, n) Dn[row] = __fadd_rn(D[row], __fmul_rn(alpha, B.yA[row]));
        if (grid_sum<2>(acc, part, &st->ticket) && threadIdx.x == 0)
        {
            st->cur = st->nxt;
            st->it = st->it + 1;
            st->finalResSum = st->resS;
            st->converged = 1;
        }
        return;
    }
    const float omega = (float)st->omega;
    auto one = [&](int row, float d, float y, float z, float sv, float t, float r0) {
        Dn[row] = __fadd_rn(d, __fadd_rn(__fmul_rn(alpha, y), __fmul_rn(omega, z)));
        const float r = __fsub_rn(sv, __fmul_rn(omega, t));
        B.rA[row] = r;
        acc[0] += (double)fabsf(r);
        acc[1] += (double)r0 * (double)r;
    };
    // rows row, row + stride, ... in that order, the loads of two issued
    // together (as k_pcg_update)
    const int stride = gridDim.x * NT;
    int row = blockIdx.x * NT + threadIdx.x;
    for (; row + stride < n; row += 2 * stride)
    {
        float d[2], y[2], z[2], sv[2], t[2], r0[2];
#pragma unroll
        for (int u = 0; u < 2; ++u)
        {
            const int i = row + u * stride;
            d[u] = D[i];
            y[u] = B.yA[i];
            z[u] = B.zA[i];
            sv[u] = B.sA[i];
            t[u] = B.tA[i];
            r0[u] = B.rA0[i];
        }
#pragma unroll
        for (int u = 0; u < 2; ++u) one(row + u * stride, d[u], y[u], z[u], sv[u], t[u], r0[u]);
    }
    for (; row < n; row += stride)
        one(row, D[row], B.yA[row], B.zA[row], B.sA[row], B.tA[row], B.rA0[row]);
    if (grid_sum<2>(acc, part, &st->ticket) && threadIdx.x == 0)
    {
        st->res = acc[0];
        st->cur = st->nxt;
        st->it = st->it + 1;
        inner_sync_point(st, false);
        st->rA0rAold = st->rA0rA;
        st->rA0rA = acc[1];
        st->beta = (st->rA0rA / st->rA0rAold) * (st->alpha / st->omega);
        if (useCond) cudaGraphSetConditional(h, st->done ? 0u : 1u);
    }
}

// ------------------------------------------------------------ test operators

// y = A x (FP32) with dot = w.y (ldu_spmv_dotw semantics, FP64 partials).
template <int MAXW, int PAIRED = 0>
static __global__ void __launch_bounds__(NT) k_spmv32(DevSell A, const float* __restrict__ diag,
                                               const float* __restrict__ x,
                                               const float* __restrict__ w,
                                               float* __restrict__ y, double* out,
                                               unsigned int* ticket, double* part)
{
    double acc[1] = {0.0};
    CF_ROWS(row, A.n)
    {
        const float v = row_f32<MAXW, PAIRED>(A, row, __fmul_rn(diag[row], x[row]),
                                      [&](int c) { return __ldg(x + c); });
        y[row] = v;
        if (w) acc[0] += (double)w[row] * (double)v;
    }
    if (grid_sum<1>(acc, part, ticket) && threadIdx.x == 0) *out = acc[0];
}

// Reads `count` float4 (an L2 flush that leaves only clean lines behind);
// the sum is stored so the loads are not removed.
static __global__ void k_read_flush(const float4* __restrict__ p, long long count, double* sink)
{
    float acc = 0.0f;
    for (long long i = (long long)blockIdx.x * NT + threadIdx.x; i < count;
         i += (long long)gridDim.x * NT)
    {
        const float4 v = __ldcg(p + i);
        acc += v.x + v.y + v.z + v.w;
    }
    if (acc == 12345.0f) *sink = acc;
}

// cheb_init (metalFoamKernels.metal:154-171), writing w0 only (z0 = w0).
static __global__ void k_cheb_init(int n, const float* __restrict__ r, const float* __restrict__ rD,
                            const float* __restrict__ chebC, float* __restrict__ w)
{
    const float c1 = chebC[0];
    CF_ROWS(row, n) w[row] = __fmul_rn(__fmul_rn(c1, rD[row]), r[row]);
}

// ------------------------------------------------- stream dispatch (host)

// The instantiation of a SpMV-carrying kernel for A: the paired stream of
// its slice width when A has one, else the column-major streams.
#define CF_PAIRED_KERNEL(A, KERNEL, ...)                                          \
    ((A).pval && (A).ellW == 4   ? KERNEL<__VA_ARGS__, 4>                         \
     : (A).pval && (A).ellW == 5 ? KERNEL<__VA_ARGS__, 5>                         \
     : (A).pval && (A).ellW == 6 ? KERNEL<__VA_ARGS__, 6>                         \
                                 : KERNEL<__VA_ARGS__, 0>)
static_assert(PAIR_MIN_W == 4 && PAIR_MAX_W == 6, "CF_PAIRED_KERNEL covers widths 4..6");

template <bool LAST>
inline auto cheb_step_kernel(const DevSell& A)
{
    return CF_PAIRED_KERNEL(A, k_cheb_step, LAST, MAXW_UNROLL);
}
inline auto spmv32_kernel(const DevSell& A) { return CF_PAIRED_KERNEL(A, k_spmv32, MAXW_UNROLL); }
inline auto pcg_p_spmv_kernel(const DevSell& A)
{
    return CF_PAIRED_KERNEL(A, k_pcg_p_spmv, MAXW_UNROLL);
}
inline auto bicg_ab_kernel(const DevSell& A) { return CF_PAIRED_KERNEL(A, k_bicg_ab, MAXW_UNROLL); }
inline auto bicg_cd_kernel(const DevSell& A) { return CF_PAIRED_KERNEL(A, k_bicg_cd, MAXW_UNROLL); }

}  // namespace cf
