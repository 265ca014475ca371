// cf_multi.cu -- several right-hand sides sharing one matrix (the
// segregated momentum components Ux, Uy, Uz of one fvMatrix).
//
// No counterpart in the reference (the design's multi-RHS row): the
// reference solves each component separately.  Here one context solves R
// (<= 4) systems A psi_r = b_r with cudaPBiCGStab semantics per component:
// every SpMV loads each matrix entry (column index and coefficient) once
// and applies it to all R vectors, every reduction carries R partial sums,
// and each component keeps its own scalars, early exit, best iterate,
// stagnation and convergence state.  Per component the arithmetic is the
// single-solve arithmetic (same row order, same operations) and every
// kernel runs on the grid of its single-solve counterpart, so each
// component's FP64 reductions fold in the same order: a multi-RHS solve
// returns bit-for-bit what R separate cf_solve calls return.
#include "cudafoam.h"
#include "cf_host.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <thread>
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
constexpr int RMAX = 4;
// components solved at once by the concurrent form (rhsTile 0)
constexpr int MAX_STREAM_COMPONENTS = 8;

struct MBufs
{
    long long n;            // stride between components
    float *rA, *rA0, *P, *yA, *AyA, *sA, *zA, *tA, *D;   // D: [3][R][n]
    double *psi, *b, *r64;
    const float* diag;
    const float* rD;
    const double* diag64;
    InnerState* st;         // [R]
    DriverState* drv;       // [R]
    double* part;
    unsigned int* ticket;
    int* active;            // components still iterating
};

// R FP32 rows sharing the entry loads; x(r, c) gives component r's x[c].
template <int R, int MAXW, class XF>
__device__ __forceinline__ void rows_f32(const DevSell& A, int row, float (&acc)[R],
                                         const bool (&on)[R], XF x)
{
    const int sl = row >> 5;
    const int b0 = __ldg(A.sliceOff + sl);
    const int w = (__ldg(A.sliceOff + sl + 1) - b0) >> 5;
    const int base = b0 + (row & 31);
    if (w <= MAXW)
    {
        int cc[MAXW];
        float v[MAXW];
#pragma unroll
        for (int k = 0; k < MAXW; ++k)
        {
            if (k < w)
            {
                cc[k] = __ldcs(A.col + base + SLICE * k);
                v[k] = __ldcs(A.val + base + SLICE * k);
            }
            else
            {
                cc[k] = -1;
                v[k] = 0.0f;
            }
        }
#pragma unroll
        for (int r = 0; r < R; ++r)
        {
            if (!on[r]) continue;
            float xv[MAXW];
#pragma unroll
            for (int k = 0; k < MAXW; ++k) xv[k] = cc[k] != -1 ? x(r, col_index(cc[k])) : 0.0f;
#pragma unroll
            for (int k = 0; k < MAXW; ++k)
                if (cc[k] != -1) acc[r] = __fadd_rn(acc[r], __fmul_rn(v[k], xv[k]));
        }
    }
    else
    {
        for (int k = 0; k < w; ++k)
        {
            const int cc = __ldcs(A.col + base + SLICE * k);
            if (cc == -1) continue;
            const float v = __ldcs(A.val + base + SLICE * k);
#pragma unroll
            for (int r = 0; r < R; ++r)
                if (on[r]) acc[r] = __fadd_rn(acc[r], __fmul_rn(v, x(r, col_index(cc))));
        }
    }
}

// R FP64 rows (Amul order) sharing the entry loads.
template <int R, int MAXW, class XF>
__device__ __forceinline__ void rows_f64(const DevSell& A, int row, double (&acc)[R],
                                         const bool (&on)[R], XF x)
{
    const int sl = row >> 5;
    const int b0 = __ldg(A.sliceOff + sl);
    const int w = (__ldg(A.sliceOff + sl + 1) - b0) >> 5;
    const int base = b0 + (row & 31);
    for (int pass = 0; pass < 2; ++pass)
    {
        for (int k = 0; k < w; ++k)
        {
            const int cc = __ldcs(A.col + base + SLICE * k);
            const bool take = pass == 0 ? is_nbr(cc) : is_own(cc);
            if (!take) continue;
            const double v = __ldcs(A.val64 + base + SLICE * k);
#pragma unroll
            for (int r = 0; r < R; ++r)
                if (on[r]) acc[r] = __dadd_rn(acc[r], __dmul_rn(v, x(r, col_index(cc))));
        }
    }
}

template <int R>
__device__ __forceinline__ void load_on(const InnerState* st, bool (&on)[R])
{
#pragma unroll
    for (int r = 0; r < R; ++r) on[r] = !st[r].done;
}

// ---------------------------------------------------------------- FP64 driver

template <int R>
__global__ void __launch_bounds__(NT) km_mean_psi(int n, MBufs M)
{
    double acc[R];
#pragma unroll
    for (int r = 0; r < R; ++r) acc[r] = 0.0;
    CF_ROWS(row, n)
    {
#pragma unroll
        for (int r = 0; r < R; ++r) acc[r] += M.psi[r * M.n + row];
    }
    if (grid_sum<R>(acc, M.part, M.ticket) && threadIdx.x == 0)
    {
#pragma unroll
        for (int r = 0; r < R; ++r) M.drv[r].xbar = acc[r] / (double)n;
    }
}

// r = b - A psi per component; with `initial` also normFactor and the
// initial residual, otherwise the normalised L1 residual of components that
// ran an inner solve (M.active).
template <int R, int MAXW>
__global__ void __launch_bounds__(NT) km_residual(DevSell A, MBufs M, const double* u,
                                                  int initial)
{
    bool on[R];
#pragma unroll
    for (int r = 0; r < R; ++r) on[r] = initial || M.active[r];
    double acc[2 * R];
#pragma unroll
    for (int r = 0; r < 2 * R; ++r) acc[r] = 0.0;
    CF_ROWS(row, A.n)
    {
        double wa[R];
#pragma unroll
        for (int r = 0; r < R; ++r) wa[r] = __dmul_rn(M.diag64[row], M.psi[r * M.n + row]);
        rows_f64<R, MAXW>(A, row, wa, on, [&](int r, int c) { return __ldg(M.psi + r * M.n + c); });
#pragma unroll
        for (int r = 0; r < R; ++r)
        {
            if (!on[r]) continue;
            const double bb = M.b[r * M.n + row];
            const double rr = __dsub_rn(bb, wa[r]);
            M.r64[r * M.n + row] = rr;
            if (initial)
            {
                const double pA = __dmul_rn(u[row], M.drv[r].xbar);
                acc[2 * r] += __dadd_rn(fabs(__dsub_rn(wa[r], pA)), fabs(__dsub_rn(bb, pA)));
            }
            acc[2 * r + 1] += fabs(rr);
        }
    }
    if (grid_sum<2 * R>(acc, M.part, M.ticket) && threadIdx.x == 0)
    {
#pragma unroll
        for (int r = 0; r < R; ++r)
        {
            if (!on[r]) continue;
            DriverState& d = M.drv[r];
            if (initial)
            {
                d.normFactor = acc[2 * r] + 1e-20;
                d.initRes = acc[2 * r + 1] / d.normFactor;
                d.finalRes = d.initRes;
            }
            else
            {
                d.finalRes = acc[2 * r + 1] / d.normFactor;
            }
        }
    }
}

// ||r_r||_2 / ||b_r||_2 (k_l2 per component)
template <int R>
__global__ void __launch_bounds__(NT) km_l2(int n, MBufs M)
{
    double acc[2 * R];
#pragma unroll
    for (int r = 0; r < 2 * R; ++r) acc[r] = 0.0;
    CF_ROWS(row, n)
    {
#pragma unroll
        for (int r = 0; r < R; ++r)
        {
            const double rr = M.r64[r * M.n + row];
            const double bb = M.b[r * M.n + row];
            acc[2 * r] += rr * rr;
            acc[2 * r + 1] += bb * bb;
        }
    }
    if (grid_sum<2 * R>(acc, M.part, M.ticket) && threadIdx.x == 0)
    {
#pragma unroll
        for (int r = 0; r < R; ++r)
        {
            M.drv[r].l2r = sqrt(acc[2 * r]);
            M.drv[r].l2b = sqrt(acc[2 * r + 1]);
        }
    }
}

// psi_r += delta_r (selected iterate), components that ran an inner solve
template <int R>
__global__ void km_psi_update(int n, MBufs M)
{
    bool on[R];
    int sel[R];
#pragma unroll
    for (int r = 0; r < R; ++r)
    {
        on[r] = M.active[r];
        sel[r] = M.st[r].sel;
    }
    CF_ROWS(row, n)
    {
#pragma unroll
        for (int r = 0; r < R; ++r)
            if (on[r])
                M.psi[r * M.n + row] = __dadd_rn(
                    M.psi[r * M.n + row],
                    (double)M.D[((size_t)sel[r] * R + r) * M.n + row]);
    }
}

// ---------------------------------------------------------------- BiCGStab

template <int R>
__global__ void km_setup(InnerState* st, const double* target, const int* maxIter, int stagLimit,
                         const int* active)
{
    const int r = threadIdx.x;
    if (r >= R || blockIdx.x != 0) return;
    InnerState& q = st[r];
    q.wArA = q.wArAold = q.wApA = q.alpha = q.beta = q.res = 0.0;
    q.rA0rA = q.rA0rAold = q.rA0AyA = q.omega = q.tAtA = q.tAsA = q.resS = 0.0;
    q.bestRes = 1.0e300;
    q.target = target[r];
    q.finalResSum = 0.0;
    q.it = 0;
    q.maxIter = maxIter[r];
    q.ips = 1;
    q.stagLimit = stagLimit > 0 ? stagLimit : STAG_LIMIT;
    q.lastSync = 0;
    q.noProgress = 0;
    q.cur = 0;
    q.best = 0;
    q.nxt = 1;
    q.converged = q.singular = q.stagnated = q.early = 0;
    q.done = (active[r] && q.maxIter > 0) ? 0 : 1;
    q.sel = 0;
    q.ticket = 0u;
}

template <int R>
__global__ void __launch_bounds__(NT) km_bicg_init(int n, MBufs M)
{
    bool on[R];
#pragma unroll
    for (int r = 0; r < R; ++r) on[r] = M.active[r];
    double acc[R];
#pragma unroll
    for (int r = 0; r < R; ++r) acc[r] = 0.0;
    CF_ROWS(row, n)
    {
#pragma unroll
        for (int r = 0; r < R; ++r)
        {
            if (!on[r]) continue;
            const size_t i = (size_t)r * M.n + row;
            const float ra = (float)M.r64[i];
            M.rA[i] = ra;
            M.rA0[i] = ra;
            M.D[i] = 0.0f;           // buffer 0 of component r
            M.P[i] = 0.0f;
            M.AyA[i] = 0.0f;
            acc[r] += (double)ra * (double)ra;
        }
    }
    if (grid_sum<R>(acc, M.part, M.ticket) && threadIdx.x == 0)
    {
#pragma unroll
        for (int r = 0; r < R; ++r)
        {
            InnerState& q = M.st[r];
            q.rA0rAold = q.rA0rA;
            q.rA0rA = acc[r];
            q.beta = 0.0;
        }
    }
}

template <int R>
__global__ void __launch_bounds__(NT) km_bicg_a(int n, MBufs M)
{
    bool on[R];
    float beta[R], omega[R];
    load_on<R>(M.st, on);
#pragma unroll
    for (int r = 0; r < R; ++r)
    {
        beta[r] = (float)M.st[r].beta;
        omega[r] = (float)M.st[r].omega;
    }
    CF_ROWS(row, n)
    {
        const float rd = M.rD[row];
#pragma unroll
        for (int r = 0; r < R; ++r)
        {
            if (!on[r]) continue;
            const size_t i = (size_t)r * M.n + row;
            const float p = __fadd_rn(M.rA[i],
                                      __fmul_rn(beta[r], __fsub_rn(M.P[i], __fmul_rn(omega[r], M.AyA[i]))));
            M.P[i] = p;
            M.yA[i] = __fmul_rn(rd, p);
        }
    }
}

template <int R, int MAXW>
__global__ void __launch_bounds__(NT) km_bicg_b(DevSell A, MBufs M)
{
    bool on[R];
    load_on<R>(M.st, on);
    double acc[R];
#pragma unroll
    for (int r = 0; r < R; ++r) acc[r] = 0.0;
    const float* __restrict__ yA = M.yA;
    CF_ROWS(row, A.n)
    {
        float y[R];
        const float dg = M.diag[row];
#pragma unroll
        for (int r = 0; r < R; ++r) y[r] = __fmul_rn(dg, yA[(size_t)r * M.n + row]);
        rows_f32<R, MAXW>(A, row, y, on, [&](int r, int c) { return __ldg(yA + (size_t)r * M.n + c); });
#pragma unroll
        for (int r = 0; r < R; ++r)
        {
            if (!on[r]) continue;
            const size_t i = (size_t)r * M.n + row;
            M.AyA[i] = y[r];
            acc[r] += (double)M.rA0[i] * (double)y[r];
        }
    }
    if (grid_sum<R>(acc, M.part, M.ticket) && threadIdx.x == 0)
    {
#pragma unroll
        for (int r = 0; r < R; ++r)
        {
            if (!on[r]) continue;
            InnerState& q = M.st[r];
            q.rA0AyA = acc[r];
            q.alpha = q.rA0rA / q.rA0AyA;
        }
    }
}

template <int R>
__global__ void __launch_bounds__(NT) km_bicg_c(int n, MBufs M, cudaGraphConditionalHandle h,
                                                int useCond)
{
    bool on[R];
    float alpha[R];
    load_on<R>(M.st, on);
#pragma unroll
    for (int r = 0; r < R; ++r) alpha[r] = (float)M.st[r].alpha;
    double acc[R];
#pragma unroll
    for (int r = 0; r < R; ++r) acc[r] = 0.0;
    CF_ROWS(row, n)
    {
        const float rd = M.rD[row];
#pragma unroll
        for (int r = 0; r < R; ++r)
        {
            if (!on[r]) continue;
            const size_t i = (size_t)r * M.n + row;
            const float sv = __fsub_rn(M.rA[i], __fmul_rn(alpha[r], M.AyA[i]));
            M.sA[i] = sv;
            M.zA[i] = __fmul_rn(rd, sv);
            acc[r] += (double)fabsf(sv);
        }
    }
    if (grid_sum<R>(acc, M.part, M.ticket) && threadIdx.x == 0)
    {
        int left = 0;
#pragma unroll
        for (int r = 0; r < R; ++r)
        {
            InnerState& q = M.st[r];
            if (on[r])
            {
                q.resS = acc[r];
                if (!isfinite(q.rA0rA) || !isfinite(q.alpha) || !isfinite(q.resS))
                {
                    q.singular = 1;
                    q.done = 1;
                }
                else if (q.resS <= q.target)
                {
                    q.early = 1;
                    q.done = 1;
                }
            }
            left += q.done ? 0 : 1;
        }
        if (useCond && left == 0) cudaGraphSetConditional(h, 0u);
    }
}

// early exits: delta += alpha yA (components flagged early in km_bicg_c, not
// yet applied); the rest: tA = A zA with sA.tA and tA.tA -> omega
template <int R, int MAXW>
__global__ void __launch_bounds__(NT) km_bicg_d(DevSell A, MBufs M)
{
    bool on[R], ear[R];
    float alpha[R];
    int cur[R], nxt[R];
#pragma unroll
    for (int r = 0; r < R; ++r)
    {
        const InnerState& q = M.st[r];
        on[r] = !q.done;
        ear[r] = q.early && !q.converged;
        alpha[r] = (float)q.alpha;
        cur[r] = q.cur;
        nxt[r] = q.nxt;
    }
    double acc[2 * R];
#pragma unroll
    for (int r = 0; r < 2 * R; ++r) acc[r] = 0.0;
    const float* __restrict__ zA = M.zA;
    CF_ROWS(row, A.n)
    {
        float t[R];
        const float dg = M.diag[row];
#pragma unroll
        for (int r = 0; r < R; ++r) t[r] = __fmul_rn(dg, zA[(size_t)r * M.n + row]);
        rows_f32<R, MAXW>(A, row, t, on, [&](int r, int c) { return __ldg(zA + (size_t)r * M.n + c); });
#pragma unroll
        for (int r = 0; r < R; ++r)
        {
            const size_t i = (size_t)r * M.n + row;
            if (on[r])
            {
                M.tA[i] = t[r];
                acc[2 * r] += (double)M.sA[i] * (double)t[r];
                acc[2 * r + 1] += (double)t[r] * (double)t[r];
            }
            else if (ear[r])
            {
                M.D[((size_t)nxt[r] * R + r) * M.n + row] =
                    __fadd_rn(M.D[((size_t)cur[r] * R + r) * M.n + row], __fmul_rn(alpha[r], M.yA[i]));
            }
        }
    }
    if (grid_sum<2 * R>(acc, M.part, M.ticket) && threadIdx.x == 0)
    {
#pragma unroll
        for (int r = 0; r < R; ++r)
        {
            InnerState& q = M.st[r];
            if (on[r])
            {
                q.tAsA = acc[2 * r];
                q.tAtA = acc[2 * r + 1];
                q.omega = q.tAsA / q.tAtA;
            }
            else if (ear[r])
            {
                q.cur = q.nxt;
                q.it = q.it + 1;
                q.finalResSum = q.resS;
                q.converged = 1;
            }
        }
    }
}

template <int R>
__global__ void __launch_bounds__(NT) km_bicg_e(int n, MBufs M, cudaGraphConditionalHandle h,
                                                int useCond)
{
    bool on[R];
    float alpha[R], omega[R];
    int cur[R], nxt[R];
#pragma unroll
    for (int r = 0; r < R; ++r)
    {
        const InnerState& q = M.st[r];
        on[r] = !q.done;
        alpha[r] = (float)q.alpha;
        omega[r] = (float)q.omega;
        cur[r] = q.cur;
        nxt[r] = q.nxt;
    }
    double acc[2 * R];
#pragma unroll
    for (int r = 0; r < 2 * R; ++r) acc[r] = 0.0;
    CF_ROWS(row, n)
    {
#pragma unroll
        for (int r = 0; r < R; ++r)
        {
            if (!on[r]) continue;
            const size_t i = (size_t)r * M.n + row;
            const float* Dc = M.D + ((size_t)cur[r] * R + r) * M.n;
            float* Dn = M.D + ((size_t)nxt[r] * R + r) * M.n;
            Dn[row] = __fadd_rn(Dc[row], __fadd_rn(__fmul_rn(alpha[r], M.yA[i]),
                                                   __fmul_rn(omega[r], M.zA[i])));
            const float rv = __fsub_rn(M.sA[i], __fmul_rn(omega[r], M.tA[i]));
            M.rA[i] = rv;
            acc[2 * r] += (double)fabsf(rv);
            acc[2 * r + 1] += (double)M.rA0[i] * (double)rv;
        }
    }
    if (grid_sum<2 * R>(acc, M.part, M.ticket) && threadIdx.x == 0)
    {
        int left = 0;
#pragma unroll
        for (int r = 0; r < R; ++r)
        {
            InnerState& q = M.st[r];
            if (on[r])
            {
                q.res = acc[2 * r];
                q.cur = q.nxt;
                q.it = q.it + 1;
                inner_sync_point(&q, false);
                q.rA0rAold = q.rA0rA;
                q.rA0rA = acc[2 * r + 1];
                q.beta = (q.rA0rA / q.rA0rAold) * (q.alpha / q.omega);
            }
            left += q.done ? 0 : 1;
        }
        if (useCond && left == 0) cudaGraphSetConditional(h, 0u);
    }
}

template <int R>
__global__ void km_final(InnerState* st, const int* active)
{
    const int r = threadIdx.x;
    if (r >= R || blockIdx.x != 0 || !active[r]) return;
    InnerState& q = st[r];
    if (q.early)
        q.sel = q.cur;
    else if (q.bestRes < q.finalResSum)
    {
        q.sel = q.best;
        q.finalResSum = q.bestRes;
    }
    else
        q.sel = q.cur;
}

}  // namespace

// ------------------------------------------------------------------ host

struct cf_multi_state
{
    int R = 0;
    long long n = 0;
    float* f = nullptr;      // all FP32 vectors
    double* d = nullptr;     // psi, b, r64
    double* part = nullptr;  // [2 RMAX][max grid] reduction partials
    InnerState* st = nullptr;
    DriverState* drv = nullptr;
    double* target = nullptr;
    int* maxIter = nullptr;
    int* active = nullptr;
    InnerState* h_st = nullptr;
    DriverState* h_drv = nullptr;
    double* h_target = nullptr;
    int* h_maxIter = nullptr;
    int* h_active = nullptr;
    std::map<int, cudaGraphExec_t> graphs;   // per R
};

namespace {

cf_multi_state* multi_state(cf_context* c)
{
    return reinterpret_cast<cf_multi_state*>(c->multi);
}

// Buffers for RMAX components of this topology; released (with the graphs,
// which hold the topology's pointers) whenever the topology is.
int ensure_multi(cf_context* c)
{
    cf_multi_state* m = multi_state(c);
    if (m && m->n == c->n) return CF_OK;
    cf_multi_release(c);
    m = new cf_multi_state();
    c->multi = m;
    m->n = c->n;
    const size_t N = (size_t)c->n * RMAX;
    // the kernels reduce up to 2 R values per launch; grid_for never returns
    // more than numSMs * maxBlocksPerSM blocks
    const size_t partCount = (size_t)2 * RMAX * c->numSMs * c->maxBlocksPerSM;
    // rA rA0 P yA AyA sA zA tA (8) + D (3)
    if (cudaMalloc((void**)&m->f, sizeof(float) * N * 11) != cudaSuccess ||
        cudaMalloc((void**)&m->d, sizeof(double) * N * 3) != cudaSuccess ||
        cudaMalloc((void**)&m->part, sizeof(double) * partCount) != cudaSuccess ||
        cudaMalloc((void**)&m->st, sizeof(InnerState) * RMAX) != cudaSuccess ||
        cudaMalloc((void**)&m->drv, sizeof(DriverState) * RMAX) != cudaSuccess ||
        cudaMalloc((void**)&m->target, sizeof(double) * RMAX) != cudaSuccess ||
        cudaMalloc((void**)&m->maxIter, sizeof(int) * RMAX) != cudaSuccess ||
        cudaMalloc((void**)&m->active, sizeof(int) * RMAX) != cudaSuccess ||
        cudaMallocHost((void**)&m->h_st, sizeof(InnerState) * RMAX) != cudaSuccess ||
        cudaMallocHost((void**)&m->h_drv, sizeof(DriverState) * RMAX) != cudaSuccess ||
        cudaMallocHost((void**)&m->h_target, sizeof(double) * RMAX) != cudaSuccess ||
        cudaMallocHost((void**)&m->h_maxIter, sizeof(int) * RMAX) != cudaSuccess ||
        cudaMallocHost((void**)&m->h_active, sizeof(int) * RMAX) != cudaSuccess)
    {
        cudaGetLastError();
        cf_multi_release(c);
        return fail(CF_ERR_CUDA, "cf_solve_multi: allocation failed");
    }
    CF_CUDA(cudaMemset(m->st, 0, sizeof(InnerState) * RMAX));
    CF_CUDA(cudaMemset(m->drv, 0, sizeof(DriverState) * RMAX));
    CF_CUDA(cudaMemset(m->f, 0, sizeof(float) * N * 11));
    return CF_OK;
}

MBufs mbufs(cf_context* c, int R)
{
    cf_multi_state* m = multi_state(c);
    const size_t N = (size_t)c->n * R;
    MBufs M;
    M.n = c->n;
    float* f = m->f;
    M.rA = f;
    M.rA0 = f + N;
    M.P = f + 2 * N;
    M.yA = f + 3 * N;
    M.AyA = f + 4 * N;
    M.sA = f + 5 * N;
    M.zA = f + 6 * N;
    M.tA = f + 7 * N;
    M.D = f + 8 * N;
    M.psi = m->d;
    M.b = m->d + N;
    M.r64 = m->d + 2 * N;
    M.diag = c->d_diag32;
    M.rD = c->d_rD32;
    M.diag64 = c->d_diag64;
    M.st = m->st;
    M.drv = m->drv;
    M.part = m->part;
    M.ticket = &c->d_drv->ticket;
    M.active = m->active;
    return M;
}

template <int R>
int launch_multi_body(cf_context* c, cudaGraphConditionalHandle h, int useCond)
{
    const DevSell A = sell_of(c);
    const MBufs M = mbufs(c, R);
    cudaStream_t s = c->stream;
    const int n = c->n;
    // grids of the single-solve kernels (same reduction order per
    // component).  The single solve fuses a into b and c into d (p, yA and
    // s, zA formed at every gathered column); here the five passes stay
    // separate -- recomputing them for every component at every gathered
    // column measured 9% slower at 64^3 x 3 -- and each pass runs on the
    // grid of the fused kernel that contains it, so every component's sums
    // fold exactly as the single solve's (the kernels it launches for this
    // layout's stream)
    const int gab = grid_for(c, (const void*)bicg_ab_kernel(A), n);
    const int gcd = grid_for(c, (const void*)bicg_cd_kernel(A), n);
    km_bicg_a<R><<<gab, NT, 0, s>>>(n, M);
    CF_LAUNCH();
    km_bicg_b<R, MW><<<gab, NT, 0, s>>>(A, M);
    CF_LAUNCH();
    km_bicg_c<R><<<gcd, NT, 0, s>>>(n, M, h, useCond);
    CF_LAUNCH();
    km_bicg_d<R, MW><<<gcd, NT, 0, s>>>(A, M);
    CF_LAUNCH();
    km_bicg_e<R><<<grid_for(c, (const void*)k_bicg_e, n), NT, 0, s>>>(n, M, h, useCond);
    CF_LAUNCH();
    return CF_OK;
}

template <int R>
int multi_graph(cf_context* c, cudaGraphExec_t* out)
{
    cf_multi_state* m = multi_state(c);
    auto it = m->graphs.find(R);
    if (it != m->graphs.end())
    {
        *out = it->second;
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
    e = cudaStreamBeginCaptureToGraph(c->stream, cp.conditional.phGraph_out[0], nullptr, nullptr,
                                      0, cudaStreamCaptureModeRelaxed);
    if (e != cudaSuccess)
    {
        cudaGraphDestroy(g);
        return fail(CF_ERR_CUDA, std::string("cudaStreamBeginCaptureToGraph: ") +
                                     cudaGetErrorString(e));
    }
    const long long before = c->launches;
    const int rc = launch_multi_body<R>(c, h, 1);
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
    m->graphs[R] = exec;
    *out = exec;
    return CF_OK;
}

bool conv_host(double tol, double relTol, double init, double fin)
{
    return (fin < tol) || (relTol > 1e-20 && fin < relTol * init);
}

// cudaPBiCGStab's driver for R components at once (metalFoamSolver.C:77-437
// with useBiCGStab: no deflation, no Chebyshev).
template <int R>
int solve_multi_R(cf_context* c, double* psi, const double* src, cudaMemcpyKind kind,
                  const cf_options* o, cf_performance* perf)
{
    CF_TRY(ensure_multi(c));
    cf_multi_state* m = multi_state(c);
    const int n = c->n;
    cudaStream_t s = c->stream;
    const DevSell A = sell_of(c);
    const MBufs M = mbufs(c, R);
    CF_CUDA(cudaEventRecord(c->ev2, s));
    // FP32 operator as cudaPBiCGStab stages it (metalFoamSolver.C:211-220)
    const int wantSym32 = c->hasLower ? 0 : 1;
    if (wantSym32 != c->val32Sym) CF_TRY(stage_vals(c, wantSym32));
    CF_TRY(stage_diag32(c, 0));
    const int g = grid_for(c, (const void*)k_gather_f64, n);
    const int gMean = grid_for(c, (const void*)k_mean_f64, n);
    const int gRes0 = grid_for(c, (const void*)k_residual0<MW>, n);
    const int gRes = grid_for(c, (const void*)k_residual<MW>, n);
    const int gInit = grid_for(c, (const void*)k_bicg_init, n);
    const int gPsi = grid_for(c, (const void*)k_psi_update, n);
    const int gL2 = grid_for(c, (const void*)k_l2, n);
    for (int r = 0; r < R; ++r)
    {
        CF_CUDA(cudaMemcpyAsync(c->d_io64, psi + (size_t)r * n, sizeof(double) * n, kind, s));
        k_gather_f64<<<g, NT, 0, s>>>(n, c->d_perm, c->d_io64, M.psi + (size_t)r * n);
        CF_LAUNCH();
        CF_CUDA(cudaMemcpyAsync(c->d_io64, src + (size_t)r * n, sizeof(double) * n, kind, s));
        k_gather_f64<<<g, NT, 0, s>>>(n, c->d_perm, c->d_io64, M.b + (size_t)r * n);
        CF_LAUNCH();
    }
    km_mean_psi<R><<<gMean, NT, 0, s>>>(n, M);
    CF_LAUNCH();
    km_residual<R, MW><<<gRes0, NT, 0, s>>>(A, M, c->d_u, 1);
    CF_LAUNCH();
    CF_CUDA(cudaMemcpyAsync(m->h_drv, m->drv, sizeof(DriverState) * R, cudaMemcpyDeviceToHost, s));
    CF_CUDA(cudaStreamSynchronize(s));
    int totalIter[R], finished[R], singular[R], stagn[R], nRest[R];
    double fr32[R];
    for (int r = 0; r < R; ++r)
    {
        cf_performance& p = perf[r];
        std::memset(&p, 0, sizeof(p));
        const DriverState& d = m->h_drv[r];
        p.normFactor = d.normFactor;
        p.initialResidual = d.initRes;
        p.finalResidual = d.initRes;
        p.chebBeta = 2.0;
        p.solved = o->minIter > 0 || !conv_host(o->tolerance, o->relTol, d.initRes, d.initRes);
        finished[r] = !p.solved;
        totalIter[r] = 0;
        singular[r] = stagn[r] = 0;
        nRest[r] = 0;
        fr32[r] = 0.0;
        m->h_target[r] = std::max(o->tolerance, o->relTol * d.initRes) * d.normFactor;
    }
    int outer = 0;
    bool all = false;
    for (outer = 0; outer <= o->maxRestarts; ++outer)
    {
        int any = 0;
        for (int r = 0; r < R; ++r)
        {
            m->h_active[r] = !finished[r];
            m->h_maxIter[r] = o->maxIter - totalIter[r];
            any |= m->h_active[r];
        }
        if (!any)
        {
            all = true;
            break;
        }
        CF_CUDA(cudaMemcpyAsync(m->target, m->h_target, sizeof(double) * R, cudaMemcpyHostToDevice, s));
        CF_CUDA(cudaMemcpyAsync(m->maxIter, m->h_maxIter, sizeof(int) * R, cudaMemcpyHostToDevice, s));
        CF_CUDA(cudaMemcpyAsync(m->active, m->h_active, sizeof(int) * R, cudaMemcpyHostToDevice, s));
        km_setup<R><<<1, 32, 0, s>>>(m->st, m->target, m->maxIter, o->stagnationLimit, m->active);
        CF_LAUNCH();
        km_bicg_init<R><<<gInit, NT, 0, s>>>(n, M);
        CF_LAUNCH();
        bool anyIter = false;
        bool graphRan = false;
        for (int r = 0; r < R; ++r) anyIter |= m->h_active[r] && m->h_maxIter[r] > 0;
        if (anyIter)
        {
            if (o->graph)
            {
                cudaGraphExec_t exec;
                CF_TRY(multi_graph<R>(c, &exec));
                CF_CUDA(cudaGraphLaunch(exec, s));
                graphRan = true;
            }
            else
            {
                for (int it = 0; it < o->maxIter; ++it)
                {
                    CF_TRY(launch_multi_body<R>(c, 0, 0));
                    CF_CUDA(cudaMemcpyAsync(m->h_st, m->st, sizeof(InnerState) * R,
                                            cudaMemcpyDeviceToHost, s));
                    CF_CUDA(cudaStreamSynchronize(s));
                    bool left = false;
                    for (int r = 0; r < R; ++r) left |= !m->h_st[r].done;
                    if (!left) break;
                }
            }
        }
        km_final<R><<<1, 32, 0, s>>>(m->st, m->active);
        CF_LAUNCH();
        km_psi_update<R><<<gPsi, NT, 0, s>>>(n, M);
        CF_LAUNCH();
        km_residual<R, MW><<<gRes, NT, 0, s>>>(A, M, c->d_u, 0);
        CF_LAUNCH();
        CF_CUDA(cudaMemcpyAsync(m->h_st, m->st, sizeof(InnerState) * R, cudaMemcpyDeviceToHost, s));
        CF_CUDA(cudaMemcpyAsync(m->h_drv, m->drv, sizeof(DriverState) * R, cudaMemcpyDeviceToHost, s));
        CF_CUDA(cudaStreamSynchronize(s));
        if (graphRan)
        {
            // five kernels per pass of the graph body, passes = longest component
            int passes = 1;
            for (int r = 0; r < R; ++r)
                if (m->h_active[r]) passes = std::max(passes, m->h_st[r].it);
            c->launches += 5LL * passes;
        }
        for (int r = 0; r < R; ++r)
        {
            if (finished[r]) continue;
            const InnerState& q = m->h_st[r];
            totalIter[r] += q.it;
            singular[r] = q.singular;
            stagn[r] = q.stagnated;
            fr32[r] = q.finalResSum;
            perf[r].finalResidual = m->h_drv[r].finalRes;
            bool stop = singular[r] || totalIter[r] >= o->maxIter;
            if (totalIter[r] >= o->minIter &&
                conv_host(o->tolerance, o->relTol, perf[r].initialResidual, perf[r].finalResidual))
                stop = true;
            if (stop)
            {
                finished[r] = 1;
                nRest[r] = outer;
            }
        }
    }
    for (int r = 0; r < R; ++r)
        if (!finished[r] && perf[r].solved) nRest[r] = o->maxRestarts + 1;
    (void)all;
    km_l2<R><<<gL2, NT, 0, s>>>(n, M);
    CF_LAUNCH();
    for (int r = 0; r < R; ++r)
    {
        k_scatter_f64<<<g, NT, 0, s>>>(n, c->d_perm, M.psi + (size_t)r * n, c->d_io64);
        CF_LAUNCH();
        CF_CUDA(cudaMemcpyAsync(psi + (size_t)r * n, c->d_io64, sizeof(double) * n,
                                kind == cudaMemcpyHostToDevice ? cudaMemcpyDeviceToHost
                                                               : cudaMemcpyDeviceToDevice, s));
    }
    CF_CUDA(cudaEventRecord(c->ev3, s));
    CF_CUDA(cudaMemcpyAsync(m->h_drv, m->drv, sizeof(DriverState) * R, cudaMemcpyDeviceToHost, s));
    CF_CUDA(cudaStreamSynchronize(s));
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, c->ev2, c->ev3);
    for (int r = 0; r < R; ++r)
    {
        cf_performance& p = perf[r];
        const DriverState& d = m->h_drv[r];
        p.residualL2 = d.l2b > 0 ? d.l2r / d.l2b : d.l2r;
        p.nIterations = totalIter[r];
        p.nRestarts = nRest[r];
        p.singular = singular[r];
        p.stagnated = stagn[r];
        p.finalResSum32 = fr32[r];
        p.converged = conv_host(o->tolerance, o->relTol, p.initialResidual, p.finalResidual);
        p.tSolve = ms * 1e-3;
    }
    return CF_OK;
}

// rhsTile 0: the components as single solves, all at once, each on a
// context of its own (cf::context_clone_matrix: this context's matrix arrays,
// its own vectors, stream and captured loops) driven from a host thread of
// its own.  Every component gets exactly what cf_solve returns for it alone.
// Solves of one component are a chain of short kernels and host
// synchronisations that leave most of the GPU idle on meshes below a few
// million cells; the concurrent chains fill it, and the matrix is stored once.
int solve_multi_streams(cf_context* c, int32_t solver, int32_t nrhs, double* psi,
                        const double* src, cudaMemcpyKind kind, const cf_options* o,
                        cf_performance* perf)
{
    const size_t n = (size_t)c->n;
    const int W = std::min<int>(nrhs, MAX_STREAM_COMPONENTS);
    while ((int)c->clones.size() < W)
    {
        cf_context* k = nullptr;
        CF_TRY(context_clone_matrix(c, &k));
        c->clones.push_back(k);
    }
    // the FP32 operator in BiCGStab's form, staged once on the shared arrays
    const int wantSym32 = c->hasLower ? 0 : 1;
    if (wantSym32 != c->val32Sym) CF_TRY(stage_vals(c, wantSym32));
    for (int w = 0; w < W; ++w) CF_TRY(context_clone_sync(c, c->clones[w]));
    // the clones' streams start after the work queued so far on this one
    CF_CUDA(cudaEventRecord(c->ev0, c->stream));
    for (int w = 0; w < W; ++w) CF_CUDA(cudaStreamWaitEvent(c->clones[w]->stream, c->ev0, 0));
    std::vector<int> rc(nrhs, CF_OK);
    std::vector<std::string> msg(nrhs);
    auto run = [&](int w) {
        for (int k = w; k < nrhs; k += W)
        {
            double* p = psi + k * n;
            const double* b = src + k * n;
            const int r = kind == cudaMemcpyHostToDevice
                              ? cf_solve(c->clones[w], solver, p, b, o, &perf[k])
                              : cf_solve_device(c->clones[w], solver, p, b, o, &perf[k]);
            if (r != CF_OK)
            {
                rc[k] = r;
                msg[k] = cf_last_error();
                return;
            }
        }
    };
    std::vector<std::thread> pool;
    std::vector<int> inlineRuns;
    for (int w = 1; w < W; ++w)
    {
        try
        {
            pool.emplace_back(run, w);
        }
        catch (...)
        {
            inlineRuns.push_back(w);   // no exception crosses the C ABI
        }
    }
    run(0);
    for (int w : inlineRuns) run(w);
    for (auto& t : pool) t.join();
    for (int k = 0; k < nrhs; ++k)
        if (rc[k] != CF_OK) return fail(rc[k], "component " + std::to_string(k) + ": " + msg[k]);
    for (int w = 0; w < W; ++w)
        c->launches += c->clones[w]->launches, c->clones[w]->launches = 0;
    return CF_OK;
}

int solve_multi(cf_context* c, int32_t solver, int32_t nrhs, double* psi, const double* src,
                cudaMemcpyKind kind, const cf_options* o, cf_performance* perf)
{
    if (!c) return fail(CF_ERR_INVALID_ARG, "context is NULL");
    if (!c->hasTopo) return fail(CF_ERR_NO_TOPOLOGY, "cf_set_topology has not been called");
    if (!c->hasCoeffs) return fail(CF_ERR_NO_COEFFS, "cf_set_coeffs has not been called");
    if (!psi || !src || !o || !perf) return fail(CF_ERR_INVALID_ARG, "NULL argument");
    if (solver != CF_SOLVER_PBICGSTAB)
        return fail(CF_ERR_UNSUPPORTED, "multi-RHS solves are cudaPBiCGStab (momentum)");
    if (o->preconditioner != CF_PRECOND_CHEBYSHEV)
        return fail(CF_ERR_UNSUPPORTED, "multi-RHS solves use the Jacobi preconditioner of "
                                        "cudaPBiCGStab (GAMG preconditions cudaPCG)");
    if (nrhs < 1) return fail(CF_ERR_INVALID_ARG, "nrhs must be >= 1");
    CF_CUDA(cudaSetDevice(c->device));
    if (c->transposed) return fail(CF_ERR_UNSUPPORTED, "transposed operator staged");
    if (c->cfgRhsTile == 0) return solve_multi_streams(c, solver, nrhs, psi, src, kind, o, perf);
    const size_t n = (size_t)c->n;
    // components per pass: the context's RHS tile (cf_set_spmv_config / cf_autotune)
    const int tile = std::max(1, std::min(RMAX, c->cfgRhsTile));
    for (int first = 0; first < nrhs; first += tile)
    {
        const int R = std::min(tile, nrhs - first);
        double* p = psi + first * n;
        const double* b = src + first * n;
        cf_performance* pf = perf + first;
        int rc = CF_OK;
        switch (R)
        {
            case 1: rc = solve_multi_R<1>(c, p, b, kind, o, pf); break;
            case 2: rc = solve_multi_R<2>(c, p, b, kind, o, pf); break;
            case 3: rc = solve_multi_R<3>(c, p, b, kind, o, pf); break;
            default: rc = solve_multi_R<4>(c, p, b, kind, o, pf); break;
        }
        if (rc != CF_OK) return rc;
    }
    return CF_OK;
}

}  // namespace

void cf_multi_release(cf_context* c)
{
    cf_multi_state* m = reinterpret_cast<cf_multi_state*>(c->multi);
    if (!m) return;
    for (auto& kv : m->graphs) cudaGraphExecDestroy(kv.second);
    cudaFree(m->f);
    cudaFree(m->d);
    cudaFree(m->part);
    cudaFree(m->st);
    cudaFree(m->drv);
    cudaFree(m->target);
    cudaFree(m->maxIter);
    cudaFree(m->active);
    cudaFreeHost(m->h_st);
    cudaFreeHost(m->h_drv);
    cudaFreeHost(m->h_target);
    cudaFreeHost(m->h_maxIter);
    cudaFreeHost(m->h_active);
    delete m;
    c->multi = nullptr;
}

extern "C" int cf_solve_multi(cf_context* c, int32_t solver, int32_t nrhs, double* psi,
                              const double* source, const cf_options* opts,
                              cf_performance* perf)
{
    return solve_multi(c, solver, nrhs, psi, source, cudaMemcpyHostToDevice, opts, perf);
}

extern "C" int cf_solve_multi_device(cf_context* c, int32_t solver, int32_t nrhs, double* psi,
                                     const double* source, const cf_options* opts,
                                     cf_performance* perf)
{
    return solve_multi(c, solver, nrhs, psi, source, cudaMemcpyDeviceToDevice, opts, perf);
}
