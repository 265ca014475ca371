// cf_amg.cu -- aggregation multigrid V-cycle as the preconditioner of the
// FP32 inner PCG (opt-in: cf_options.preconditioner = CF_PRECOND_GAMG).
//
// The reference has no such preconditioner (README.md:221-227 names GAMG
// as a limitation of the Metal path); the driver around the inner solve
// (FP64 residual, deflation, restarts, polish) is unchanged.  Only the
// preconditioner apply z = M r of metalFoamBackend::pcg changes: the
// Chebyshev-Jacobi polynomial (.C:342-385) is replaced by one symmetric
// V-cycle, so PCG keeps a fixed SPD preconditioner.
//
// Hierarchy (built once per topology on the host, by the first GAMG solve):
// level 0 is the context's matrix in its internal row order.  Each level's
// cells are grouped into aggregates by root-based greedy aggregation along
// the strong couplings of that solve's coefficients (a cell whose strong
// neighbours are all free becomes a root and takes up to 7 of them; the others join
// the aggregate they are most strongly coupled to); the aggregates,
// numbered in the order their roots are met, are the next level's cells.
// Later solves keep the hierarchy and re-sum its operators.  The
// coarse operator is the Galerkin product P^T A P with the piecewise
// constant P: a coarse face sums the fine faces between its two
// aggregates, a coarse diagonal sums its cells' diagonals and twice the
// faces inside it.  Coefficients are summed on the device for every solve
// (segment sums in a fixed order, FP64), so a coefficient change needs no
// host work.  The coarsest level (at most 128 cells) is inverted densely
// (Gauss-Jordan, FP64) once per solve.
//
// V-cycle on level l (b = the level's right-hand side):
//   x  = S(b)                  Chebyshev-Jacobi from 0 (degree nSweeps on
//                              level 0, 2 below)
//   r  = b - A x;  b' = P^T r;  x' = V-cycle(l+1, b');  x += a P x'
//   x += S(b - A x)            the same polynomial (symmetric cycle)
// a = scaleCorrection, fixed in (0, 2), so the cycle is a fixed SPD
// operator.  The smoother's interval is [beta/ratio, beta] with beta the
// Gershgorin bound of D^-1 A on level 0 (metalFoamSolver.C:229-249) and
// ratio the smootherRatio control (default 8); Galerkin levels of a diagonally
// dominant matrix with non-positive off-diagonals keep that bound.  Level 0
// reuses the Krylov kernels (its pre-smoother start w0 = c1 rD r is formed
// by the update kernel, its last post-smoothing step forms z.r and beta).
// The restriction is formed by the kernel that starts the next level, and
// the prolongation by the first post-smoothing step, which reads x + a P x'
// on the fly, so a coarse level costs five launches.
#include "cudafoam.h"
#include "cf_host.hpp"

#include <algorithm>
#include <cstdio>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "cf_kernels.cuh"

using namespace cf;

#define AMG_CUDA(call)                                                          \
    do                                                                          \
    {                                                                           \
        cudaError_t e_ = (call);                                                \
        if (e_ != cudaSuccess)                                                  \
            return fail(CF_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define AMG_TRY(expr)                 \
    do                                \
    {                                 \
        int rc_ = (expr);             \
        if (rc_ != CF_OK) return rc_; \
    } while (0)

#define AMG_LAUNCH()                                                            \
    do                                                                          \
    {                                                                           \
        cudaError_t e_ = cudaGetLastError();                                    \
        if (e_ != cudaSuccess)                                                  \
            return fail(CF_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e_)); \
        c->launches++;                                                          \
    } while (0)

namespace cf {

constexpr int AMG_MAX_COARSEST = 128;
constexpr int AMG_MAX_LEVELS = 16;
constexpr int AMG_INV_THREADS = 1024;
constexpr int AMG_MAX_AGG = 8;       // cells per root aggregate at most
constexpr double AMG_STRONG = 0.08;  // strong coupling: |a_ij| >= this * sqrt(a_ii a_jj)
constexpr int AMG_COARSE_DEGREE = 2; // smoother degree below level 0 (at most nSweeps)

struct AmgLevel
{
    int n = 0;
    int nf = 0;                 // faces of this level (coarse levels: between aggregates)
    // operator (levels >= 1; level 0 is the context's own)
    DevSell A;
    float* diag32 = nullptr;
    float* rD32 = nullptr;
    double* upper64 = nullptr;  // [nf] face coefficients (FP64)
    double* diag64 = nullptr;   // [n]
    int* eface = nullptr;       // SELL entry -> face
    long long nnzp = 0;
    // work vectors (levels >= 1)
    float* b = nullptr;
    float* x0 = nullptr;
    float* x1 = nullptr;
    float* w = nullptr;
    float* r = nullptr;
    // to the next level (absent on the coarsest)
    int nagg = 0;
    int* agg = nullptr;         // [n] aggregate of each row
    int* aggStart = nullptr;    // [nagg + 1]
    int* aggRows = nullptr;     // [n] rows by aggregate, ascending
    int* cfStart = nullptr;     // [nf(l+1) + 1] this level's faces of each coarse face
    int* cfList = nullptr;
    int* intStart = nullptr;    // [nagg + 1] this level's faces inside each aggregate
    int* intList = nullptr;
    // host copies for cf_gamg_export: this level's faces (levels >= 1) and
    // the aggregate of each row (levels with a coarser one)
    std::vector<int> hLow, hUpp, hAgg;
};

struct AmgData
{
    int coarsestCap = 0;        // nCellsInCoarsestLevel the hierarchy was built for
    std::vector<AmgLevel> lv;
    std::vector<void*> allocs;
    double* coarseInv = nullptr;   // [nc * nc] inverse of the coarsest operator (row-major)
    float* scale = nullptr;        // scaleCorrection of the current solve
    float hostScale = 1.0f;        // its host copy (source of the async upload)
};

namespace {

template <class T>
int amg_alloc(cf_context* c, AmgData* d, T** p, size_t count)
{
    *p = nullptr;
    if (count == 0) count = 1;
    const cudaError_t e = cudaMalloc((void**)p, count * sizeof(T));
    if (e != cudaSuccess)
        return fail(CF_ERR_CUDA, std::string("cudaMalloc (multigrid): ") + cudaGetErrorString(e));
    d->allocs.push_back((void*)*p);
    (void)c;
    return CF_OK;
}

template <class T>
int amg_upload(cf_context* c, AmgData* d, T** p, const std::vector<T>& h)
{
    AMG_TRY(amg_alloc(c, d, p, h.size()));
    if (!h.empty())
        AMG_CUDA(cudaMemcpyAsync(*p, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice,
                                 c->stream));
    return CF_OK;
}

// Root-based greedy aggregation of the cell graph (CSR adjacency) guided by
// the coupling strength s_ij = |a_ij| / sqrt(a_ii a_jj) of each edge: a
// cell with at least one strong edge (s_ij >= AMG_STRONG) whose strong
// neighbours are all free becomes a root and takes its free strong
// neighbours, at most AMG_MAX_AGG - 1 of them (so coarse levels, whose
// graphs are denser, still coarsen by about 8 per level); every other cell
// joins the aggregated neighbour it is most strongly coupled to.  Strong
// edges keep cells that are tightly coupled (large coefficients) together,
// which a piecewise constant interpolation needs on heterogeneous media.
int aggregate(int n, const std::vector<int>& xadj, const std::vector<int>& adj,
              const std::vector<double>& str, std::vector<int>& agg)
{
    agg.assign(n, -1);
    int nagg = 0;
    for (int i = 0; i < n; ++i)
    {
        if (agg[i] >= 0) continue;
        bool free = true;
        bool anyStrong = false;
        for (int q = xadj[i]; q < xadj[i + 1] && free; ++q)
            if (str[q] >= AMG_STRONG)
            {
                anyStrong = true;
                free = agg[adj[q]] < 0;
            }
        if (!free || !anyStrong) continue;
        agg[i] = nagg;
        int taken = 1;
        for (int q = xadj[i]; q < xadj[i + 1] && taken < AMG_MAX_AGG; ++q)
            if (str[q] >= AMG_STRONG && agg[adj[q]] < 0)
            {
                agg[adj[q]] = nagg;
                ++taken;
            }
        ++nagg;
    }
    // the rest join their most strongly coupled aggregated neighbour
    // (decided against the root phase's assignment only)
    std::vector<int> join(n, -1);
    for (int i = 0; i < n; ++i)
    {
        if (agg[i] >= 0) continue;
        double best = -1.0;
        for (int q = xadj[i]; q < xadj[i + 1]; ++q)
            if (agg[adj[q]] >= 0 && str[q] > best)
            {
                best = str[q];
                join[i] = agg[adj[q]];
            }
    }
    for (int i = 0; i < n; ++i)
        if (agg[i] < 0 && join[i] >= 0) agg[i] = join[i];
    // cells with no aggregated neighbour: new aggregates with their free neighbours
    for (int i = 0; i < n; ++i)
    {
        if (agg[i] >= 0) continue;
        agg[i] = nagg;
        int taken = 1;
        for (int q = xadj[i]; q < xadj[i + 1] && taken < AMG_MAX_AGG; ++q)
            if (agg[adj[q]] < 0)
            {
                agg[adj[q]] = nagg;
                ++taken;
            }
        ++nagg;
    }
    return nagg;
}

void csr_of_faces(int n, const std::vector<int>& lo, const std::vector<int>& up,
                  std::vector<int>& xadj, std::vector<int>& adj, std::vector<int>& adjFace)
{
    xadj.assign(n + 1, 0);
    for (size_t f = 0; f < lo.size(); ++f)
    {
        ++xadj[lo[f] + 1];
        ++xadj[up[f] + 1];
    }
    for (int i = 0; i < n; ++i) xadj[i + 1] += xadj[i];
    adj.assign(xadj[n], 0);
    adjFace.assign(xadj[n], 0);
    std::vector<int> pos(xadj.begin(), xadj.end() - 1);
    for (size_t f = 0; f < lo.size(); ++f)
    {
        adjFace[pos[lo[f]]] = (int)f;
        adj[pos[lo[f]]++] = up[f];
        adjFace[pos[up[f]]] = (int)f;
        adj[pos[up[f]]++] = lo[f];
    }
}

// ---------------------------------------------------------------- kernels

// coarse face coefficient: the sum of the fine faces between its aggregates
__global__ void ka_coarse_upper(int nfc, const int* __restrict__ start, const int* __restrict__ list,
                                const double* __restrict__ upper, double* __restrict__ out)
{
    for (int F = blockIdx.x * NT + threadIdx.x; F < nfc; F += gridDim.x * NT)
    {
        double s = 0.0;
        for (int q = start[F]; q < start[F + 1]; ++q) s += upper[list[q]];
        out[F] = s;
    }
}

// coarse diagonal: the cells' diagonals plus both sides of the inner faces.
// Level 0's diagonal is diag64 - u when the driver deflates (the staged
// FP32 operator of metalFoamSolver.C:197-209).
__global__ void ka_coarse_diag(int nagg, const int* __restrict__ aggStart,
                               const int* __restrict__ aggRows, const int* __restrict__ intStart,
                               const int* __restrict__ intList, const double* __restrict__ diag,
                               const double* __restrict__ u, int deflate,
                               const double* __restrict__ upper, double* __restrict__ out64,
                               float* __restrict__ out32, float* __restrict__ rD32)
{
    for (int K = blockIdx.x * NT + threadIdx.x; K < nagg; K += gridDim.x * NT)
    {
        double s = 0.0;
        for (int q = aggStart[K]; q < aggStart[K + 1]; ++q)
        {
            const int i = aggRows[q];
            s += deflate ? __dsub_rn(diag[i], u[i]) : diag[i];
        }
        for (int q = intStart[K]; q < intStart[K + 1]; ++q) s += 2.0 * upper[intList[q]];
        out64[K] = s;
        out32[K] = (float)s;
        rD32[K] = (float)(1.0 / s);
    }
}

// symmetric SELL values of a coarse level
__global__ void ka_stage_vals(long long nnzp, const int* __restrict__ eface,
                              const double* __restrict__ upper, float* __restrict__ val)
{
    for (long long e = (long long)blockIdx.x * NT + threadIdx.x; e < nnzp;
         e += (long long)gridDim.x * NT)
    {
        const int f = eface[e];
        val[e] = f < 0 ? 0.0f : (float)upper[f];
    }
}

// Dense coarsest operator (+ s 11^T when it is singular by construction)
// and its inverse, one block: the matrix lives in shared memory and is
// inverted in place by Gauss-Jordan without pivoting (SPD), then written out.
__global__ void __launch_bounds__(AMG_INV_THREADS)
    ka_coarse_invert(int nc, const int* __restrict__ sliceOff, const int* __restrict__ col,
                     const int* __restrict__ eface, const double* __restrict__ upper,
                     const double* __restrict__ diag, int shift, double* __restrict__ inv)
{
    extern __shared__ double sm[];
    double* M = sm;               // nc * nc
    double* colp = sm + nc * nc;  // column p of the current step
    const int t = threadIdx.x;
    const int nn = nc * nc;
    double dsum = 0.0;
    for (int i = 0; i < nc; ++i) dsum += diag[i];
    const double s = shift ? dsum / ((double)nc * (double)nc) : 0.0;
    for (int k = t; k < nn; k += blockDim.x) M[k] = s;
    __syncthreads();
    for (int i = t; i < nc; i += blockDim.x)
    {
        M[i * nc + i] += diag[i];
        const int sl = i / SLICE;
        const int w = (sliceOff[sl + 1] - sliceOff[sl]) / SLICE;
        for (int k = 0; k < w; ++k)
        {
            const int e = sliceOff[sl] + SLICE * k + (i % SLICE);
            const int cc = col[e];
            if (cc == -1) continue;
            M[i * nc + col_index(cc)] += upper[eface[e]];
        }
    }
    __syncthreads();
    for (int p = 0; p < nc; ++p)
    {
        const double pinv = 1.0 / M[p * nc + p];
        for (int i = t; i < nc; i += blockDim.x) colp[i] = M[i * nc + p];
        __syncthreads();
        for (int j = t; j < nc; j += blockDim.x)
            M[p * nc + j] = (j == p) ? pinv : M[p * nc + j] * pinv;
        __syncthreads();
        for (int k = t; k < nn; k += blockDim.x)
        {
            const int i = k / nc;
            if (i == p) continue;
            const int j = k - i * nc;
            M[k] = ((j == p) ? 0.0 : M[k]) - M[p * nc + j] * colp[i];
        }
        __syncthreads();
    }
    for (int k = t; k < nn; k += blockDim.x) inv[k] = M[k];
}

// The coarsest level: b = P^T r (per aggregate, its rows in ascending
// order) and x = inv b, one block (a warp per row of the GEMV: coalesced
// loads, fixed shuffle tree).
__global__ void __launch_bounds__(AMG_INV_THREADS)
    ka_restrict_coarse_solve(int nc, const int* __restrict__ aggStart,
                             const int* __restrict__ aggRows, const float* __restrict__ r,
                             const double* __restrict__ inv, float* __restrict__ b,
                             float* __restrict__ x, const InnerState* st)
{
    __shared__ float sb[AMG_MAX_COARSEST];
    if (st->done) return;
    for (int k = threadIdx.x; k < nc; k += AMG_INV_THREADS)
    {
        float acc = 0.0f;
        for (int q = aggStart[k]; q < aggStart[k + 1]; ++q) acc = __fadd_rn(acc, r[aggRows[q]]);
        sb[k] = acc;
        b[k] = acc;
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    for (int i = warp; i < nc; i += AMG_INV_THREADS / 32)
    {
        double acc = 0.0;
        for (int j = lane; j < nc; j += 32) acc += inv[i * nc + j] * (double)sb[j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) x[i] = (float)acc;
    }
}

// Off-diagonal part of a coarse row, formed by T lanes together: lane
// `sub` takes entries sub, sub + T, ... (up to four loads in flight), the
// T partial sums are combined by a fixed shuffle tree.  Every lane of the
// warp must call it (rows past the end pass valid = false).
template <int T, class XF>
__device__ __forceinline__ float row_coarse_lanes(const DevSell& A, int row, bool valid, int sub,
                                                  XF xf)
{
    float acc = 0.0f;
    if (valid)
    {
        const int sl = row >> 5;
        const int b0 = A.ellW ? sl * SLICE * A.ellW : __ldg(A.sliceOff + sl);
        const int w = A.ellW ? A.ellW : (__ldg(A.sliceOff + sl + 1) - b0) >> 5;
        const int base = b0 + (row & 31);
        for (int k0 = sub; k0 < w; k0 += 4 * T)
        {
            int c[4];
            float v[4];
#pragma unroll
            for (int q = 0; q < 4; ++q)
            {
                const int k = k0 + q * T;
                if (k < w)
                {
                    c[q] = __ldcs(A.col + base + SLICE * k);
                    v[q] = __ldcs(A.val + base + SLICE * k);
                }
                else
                {
                    c[q] = -1;
                    v[q] = 0.0f;
                }
            }
            float x[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) x[q] = (c[q] != -1) ? xf(col_index(c[q])) : 0.0f;
#pragma unroll
            for (int q = 0; q < 4; ++q)
                if (c[q] != -1) acc = __fadd_rn(acc, __fmul_rn(v[q], x[q]));
        }
    }
#pragma unroll
    for (int o = T / 2; o > 0; o >>= 1) acc = __fadd_rn(acc, __shfl_xor_sync(0xffffffffu, acc, o));
    return acc;
}

// b = P^T r (per aggregate, its rows in ascending order) and the start of
// the level's pre-smoothing from zero, x = w = c1 rD b
__global__ void __launch_bounds__(NT) ka_restrict_init(int n, const int* __restrict__ aggStart,
                                                       const int* __restrict__ aggRows,
                                                       const float* __restrict__ r,
                                                       const float* __restrict__ rD,
                                                       const float* __restrict__ cc,
                                                       float* __restrict__ b, float* __restrict__ x,
                                                       float* __restrict__ w, const InnerState* st)
{
    if (st->done) return;
    const float c1 = cc[0];
    CF_ROWS(row, n)
    {
        float acc = 0.0f;
        for (int q = aggStart[row]; q < aggStart[row + 1]; ++q) acc = __fadd_rn(acc, r[aggRows[q]]);
        b[row] = acc;
        const float v = __fmul_rn(__fmul_rn(c1, rD[row]), acc);
        x[row] = v;
        w[row] = v;
    }
}

// The iterate a smoothing step starts from: xin, or with PROLONG the
// prolonged xin + a xc[agg] (the coarse-grid correction applied on the fly,
// rounded as a separate update would be).
template <bool PROLONG>
struct StartX
{
    const float* xin;
    const int* agg;
    const float* xc;
    float a;
    __device__ __forceinline__ float operator()(int q) const
    {
        if (!PROLONG) return __ldg(xin + q);
        return __fadd_rn(__ldg(xin + q), __fmul_rn(a, __ldg(xc + __ldg(agg + q))));
    }
};

// Chebyshev step j >= 1:  w = c2 w + c3 rD (b - A xin);  xout = xin + w.
// j = 0 starts the post-smoother from xin:  w = c1 rD (b - A xin).
template <int MAXW, bool PROLONG>
__global__ void __launch_bounds__(NT) ka_step(DevSell A, const float* __restrict__ diag,
                                              const float* __restrict__ rD,
                                              const float* __restrict__ b, const float* xin,
                                              const int* __restrict__ agg, const float* xc,
                                              const float* __restrict__ scale, float* w,
                                              float* xout, const float* __restrict__ cc, int j,
                                              const InnerState* st)
{
    if (st->done) return;
    const float c2 = j > 0 ? cc[2 * j - 1] : 0.0f;
    const float c3 = j > 0 ? cc[2 * j] : cc[0];
    const StartX<PROLONG> xf{xin, agg, xc, PROLONG ? *scale : 0.0f};
    CF_ROWS(row, A.n)
    {
        const float xr = xf(row);
        const float v = row_f32<MAXW>(A, row, __fmul_rn(diag[row], xr), xf);
        const float s = __fmul_rn(__fmul_rn(c3, rD[row]), __fsub_rn(b[row], v));
        const float wn = j > 0 ? __fadd_rn(__fmul_rn(c2, w[row]), s) : s;
        w[row] = wn;
        xout[row] = __fadd_rn(xr, wn);
    }
}

// r = b - A x
template <int MAXW>
__global__ void __launch_bounds__(NT) ka_resid(DevSell A, const float* __restrict__ diag,
                                               const float* __restrict__ b,
                                               const float* __restrict__ x, float* __restrict__ r,
                                               const InnerState* st)
{
    if (st->done) return;
    CF_ROWS(row, A.n)
    {
        const float v = row_f32<MAXW>(A, row, __fmul_rn(diag[row], x[row]),
                                      [&](int q) { return __ldg(x + q); });
        r[row] = __fsub_rn(b[row], v);
    }
}

// The coarse-level step and residual with T lanes per row: 8 on levels of
// fewer than AMG_LANES8_ROWS cells, where one thread per row is
// latency-bound, 2 on larger coarse levels (measured faster than 1, 4 or 8
// there).
constexpr int AMG_LANES8_ROWS = 100000;

template <bool RESID, int T, bool PROLONG>
__global__ void __launch_bounds__(NT) ka_step_lanes(DevSell A, const float* __restrict__ diag,
                                                    const float* __restrict__ rD,
                                                    const float* __restrict__ b, const float* xin,
                                                    const int* __restrict__ agg, const float* xc,
                                                    const float* __restrict__ scale, float* w,
                                                    float* xout, const float* __restrict__ cc,
                                                    int j, const InnerState* st)
{
    if (st->done) return;
    const int lane = threadIdx.x & 31;
    const int sub = lane & (T - 1);
    const int warpG = (blockIdx.x * NT + threadIdx.x) >> 5;
    const int warps = gridDim.x * (NT / 32);
    const float c2 = j > 0 ? cc[2 * j - 1] : 0.0f;
    const float c3 = j > 0 ? cc[2 * j] : cc[0];
    const StartX<PROLONG> xf{xin, agg, xc, PROLONG ? *scale : 0.0f};
    for (int r0 = warpG * (32 / T); r0 < A.n; r0 += warps * (32 / T))
    {
        const int row = r0 + lane / T;
        const bool valid = row < A.n;
        const float off = row_coarse_lanes<T>(A, row, valid, sub, xf);
        if (valid && sub == 0)
        {
            const float xr = xf(row);
            const float v = __fadd_rn(__fmul_rn(diag[row], xr), off);
            if (RESID)
            {
                xout[row] = __fsub_rn(b[row], v);   // r = b - A x
            }
            else
            {
                const float s = __fmul_rn(__fmul_rn(c3, rD[row]), __fsub_rn(b[row], v));
                const float wn = j > 0 ? __fadd_rn(__fmul_rn(c2, w[row]), s) : s;
                w[row] = wn;
                xout[row] = __fadd_rn(xr, wn);
            }
        }
    }
}



constexpr int MW = MAXW_UNROLL;

int grid_n(cf_context* c, const void* fn, long long n) { return grid_for(c, fn, n); }

// A Chebyshev step (j; 0 starts from xin, prolonged on the fly when xc is
// given) or the residual (resid) of a coarse level with the lane-parallel
// rows.
int launch_lanes(cf_context* c, AmgData* d, const AmgLevel& L, bool resid, const float* xin,
                 const float* xc, float* xout, int j)
{
    cudaStream_t s = c->stream;
    const InnerState* st = c->d_st;
    const float* cc = c->d_chebC;
    float* w = resid ? nullptr : L.w;
    const int* agg = L.agg;
    const float* sc = d->scale;
#define AMG_LANES_LAUNCH(RES, T, PRO)                                                        \
    ka_step_lanes<RES, T, PRO><<<grid_n(c, (const void*)ka_step_lanes<RES, T, PRO>,          \
                                        (long long)L.n * T),                                   \
                                 NT, 0, s>>>(L.A, L.diag32, L.rD32, L.b, xin, agg, xc, sc, w, \
                                             xout, cc, j, st)
    const bool pro = xc != nullptr;
    if (L.n < AMG_LANES8_ROWS)
    {
        if (resid)
            AMG_LANES_LAUNCH(true, 8, false);
        else if (pro)
            AMG_LANES_LAUNCH(false, 8, true);
        else
            AMG_LANES_LAUNCH(false, 8, false);
    }
    else
    {
        if (resid)
            AMG_LANES_LAUNCH(true, 2, false);
        else if (pro)
            AMG_LANES_LAUNCH(false, 2, true);
        else
            AMG_LANES_LAUNCH(false, 2, false);
    }
#undef AMG_LANES_LAUNCH
    AMG_LAUNCH();
    return CF_OK;
}

// Level l >= 1 of the V-cycle on its own buffers, from the residual rf of
// level l - 1 (restricted here); returns the buffer holding the level's
// correction, still to be prolonged by the caller.
int vcycle_coarse(cf_context* c, AmgData* d, int l, int degree, const float* rf, float** result)
{
    AmgLevel& L = d->lv[l];
    const AmgLevel& F = d->lv[l - 1];
    cudaStream_t s = c->stream;
    const InnerState* st = c->d_st;
    const int last = (int)d->lv.size() - 1;
    if (l == last)
    {
        ka_restrict_coarse_solve<<<1, AMG_INV_THREADS, 0, s>>>(L.n, F.aggStart, F.aggRows, rf,
                                                               d->coarseInv, L.b, L.x0, st);
        AMG_LAUNCH();
        *result = L.x0;
        return CF_OK;
    }
    // right-hand side and pre-smoothing from zero
    ka_restrict_init<<<grid_n(c, (const void*)ka_restrict_init, L.n), NT, 0, s>>>(
        L.n, F.aggStart, F.aggRows, rf, L.rD32, c->d_chebC, L.b, L.x0, L.w, st);
    AMG_LAUNCH();
    float* xa = L.x0;
    float* xb = L.x1;
    for (int j = 1; j < degree; ++j)
    {
        AMG_TRY(launch_lanes(c, d, L, false, xa, nullptr, xb, j));
        std::swap(xa, xb);
    }
    // coarse-grid correction
    AMG_TRY(launch_lanes(c, d, L, true, xa, nullptr, L.r, 0));
    float* xc = nullptr;
    AMG_TRY(vcycle_coarse(c, d, l + 1, degree, L.r, &xc));
    // post-smoothing from x + a P x'
    for (int j = 0; j < degree; ++j)
    {
        AMG_TRY(launch_lanes(c, d, L, false, xa, j == 0 ? xc : nullptr, xb, j));
        std::swap(xa, xb);
    }
    *result = xa;
    return CF_OK;
}

}  // namespace

void amg_release(cf_context* c)
{
    AmgData* d = static_cast<AmgData*>(c->amg);
    if (!d) return;
    for (void* p : d->allocs) cudaFree(p);
    delete d;
    c->amg = nullptr;
}

int amg_levels(const cf_context* c)
{
    const AmgData* d = static_cast<const AmgData*>(c->amg);
    return d ? (int)d->lv.size() : 0;
}

int amg_level_cells(const cf_context* c, int l)
{
    const AmgData* d = static_cast<const AmgData*>(c->amg);
    return (d && l >= 0 && l < (int)d->lv.size()) ? d->lv[l].n : 0;
}

// Hierarchy of the context's topology (host aggregation, device layouts).
int amg_prepare(cf_context* c, int coarsestCap, bool profile)
{
    AmgData* old = static_cast<AmgData*>(c->amg);
    if (old && old->coarsestCap == coarsestCap) return CF_OK;
    amg_release(c);
    AmgData* d = new AmgData();
    c->amg = d;
    d->coarsestCap = coarsestCap;
    const double t0 = wall_now();
    double tAgg = 0.0, tCoarse = 0.0, tLayout = 0.0;
    const int n = c->n;
    const int nf = c->nf;
    // level-0 faces in the internal row order (the caller's face order kept,
    // so face f addresses the caller's upper[f])
    std::vector<int> lo(nf), up(nf);
    if (nf > 0)
    {
        AMG_CUDA(cudaMemcpyAsync(lo.data(), c->d_low, sizeof(int) * nf, cudaMemcpyDeviceToHost,
                                 c->stream));
        AMG_CUDA(cudaMemcpyAsync(up.data(), c->d_upp, sizeof(int) * nf, cudaMemcpyDeviceToHost,
                                 c->stream));
        AMG_CUDA(cudaStreamSynchronize(c->stream));
    }
    {
        std::vector<int> iperm(n);
        for (int r = 0; r < n; ++r) iperm[c->perm[r]] = r;
        for (int f = 0; f < nf; ++f)
        {
            lo[f] = iperm[lo[f]];
            up[f] = iperm[up[f]];
        }
    }
    // the coefficients the aggregation is guided by: those staged for this
    // solve (internal-order diagonal, caller-order faces); later solves with
    // other coefficients keep the hierarchy and re-sum its operators
    std::vector<double> hd(n), hu(nf);
    AMG_CUDA(cudaMemcpyAsync(hd.data(), c->d_diag64, sizeof(double) * n, cudaMemcpyDeviceToHost,
                             c->stream));
    if (nf > 0)
        AMG_CUDA(cudaMemcpyAsync(hu.data(), c->d_upper, sizeof(double) * nf,
                                 cudaMemcpyDeviceToHost, c->stream));
    AMG_CUDA(cudaStreamSynchronize(c->stream));
    d->lv.emplace_back();
    d->lv[0].n = n;
    d->lv[0].nf = nf;
    int cur = 0;
    // (at least one coarse level, also for meshes already below the cap)
    while ((int)d->lv.size() < AMG_MAX_LEVELS &&
           (d->lv[cur].n > coarsestCap || d->lv.size() == 1))
    {
        const int nl = d->lv[cur].n;
        const int nfl = (int)lo.size();
        const double ta = wall_now();
        std::vector<int> xadj, adj, adjFace, agg;
        csr_of_faces(nl, lo, up, xadj, adj, adjFace);
        std::vector<double> str(adj.size());
        for (int i = 0; i < nl; ++i)
            for (int q = xadj[i]; q < xadj[i + 1]; ++q)
            {
                const double dd = std::fabs(hd[i]) * std::fabs(hd[adj[q]]);
                str[q] = dd > 0.0 ? std::fabs(hu[adjFace[q]]) / std::sqrt(dd) : 0.0;
            }
        const int nagg = aggregate(nl, xadj, adj, str, agg);
        const double tb = wall_now();
        tAgg += tb - ta;
        if (nagg >= nl || nagg < 1) break;   // no coarsening possible
        // members of each aggregate (ascending rows)
        std::vector<int> aggStart(nagg + 1, 0), aggRows(nl);
        for (int i = 0; i < nl; ++i) ++aggStart[agg[i] + 1];
        for (int k = 0; k < nagg; ++k) aggStart[k + 1] += aggStart[k];
        {
            std::vector<int> pos(aggStart.begin(), aggStart.end() - 1);
            for (int i = 0; i < nl; ++i) aggRows[pos[agg[i]]++] = i;
        }
        // faces inside aggregates, and coarse faces (owner < neighbour, sorted)
        std::vector<int> intStart(nagg + 1, 0), intList;
        // faces between aggregates, grouped by their lower aggregate
        // (counting sort), then each group ordered by (upper aggregate,
        // face): the order of a full sort by (pair, face), in linear time
        std::vector<int> bstart(nagg + 1, 0);
        for (int f = 0; f < nfl; ++f)
        {
            const int a = agg[lo[f]];
            const int b = agg[up[f]];
            if (a == b)
                ++intStart[a + 1];
            else
                ++bstart[std::min(a, b) + 1];
        }
        for (int k = 0; k < nagg; ++k) bstart[k + 1] += bstart[k];
        std::vector<std::pair<int, int>> between(bstart[nagg]);   // (upper aggregate, face)
        {
            std::vector<int> pos(bstart.begin(), bstart.end() - 1);
            for (int f = 0; f < nfl; ++f)
            {
                const int a = agg[lo[f]];
                const int b = agg[up[f]];
                if (a != b) between[pos[std::min(a, b)]++] = {std::max(a, b), f};
            }
        }
        for (int k = 0; k < nagg; ++k)
            std::sort(between.begin() + bstart[k], between.begin() + bstart[k + 1]);
        for (int k = 0; k < nagg; ++k) intStart[k + 1] += intStart[k];
        intList.assign(intStart[nagg], 0);
        {
            std::vector<int> pos(intStart.begin(), intStart.end() - 1);
            for (int f = 0; f < nfl; ++f)
            {
                const int a = agg[lo[f]];
                if (a == agg[up[f]]) intList[pos[a]++] = f;
            }
        }
        std::vector<int> clo, cup, cfStart, cfList(between.size());
        for (int k = 0; k < nagg; ++k)
            for (int q = bstart[k]; q < bstart[k + 1]; ++q)
            {
                if (q == bstart[k] || between[q].first != between[q - 1].first)
                {
                    cfStart.push_back(q);
                    clo.push_back(k);
                    cup.push_back(between[q].first);
                }
                cfList[q] = between[q].second;
            }
        cfStart.push_back((int)between.size());
        const int nfc = (int)clo.size();
        const double tc = wall_now();
        tCoarse += tc - tb;

        AmgLevel& L = d->lv[cur];
        L.nagg = nagg;
        L.hAgg = agg;
        AMG_TRY(amg_upload(c, d, &L.agg, agg));
        AMG_TRY(amg_upload(c, d, &L.aggStart, aggStart));
        AMG_TRY(amg_upload(c, d, &L.aggRows, aggRows));
        AMG_TRY(amg_upload(c, d, &L.intStart, intStart));
        AMG_TRY(amg_upload(c, d, &L.intList, intList));
        AMG_TRY(amg_upload(c, d, &L.cfStart, cfStart));
        AMG_TRY(amg_upload(c, d, &L.cfList, cfList));

        // the coarse level's LDU addressing and SELL layout (identity order)
        std::vector<int> own(nagg + 1, 0), losS(nagg + 1, 0), los(nfc);
        for (int F = 0; F < nfc; ++F)
        {
            ++own[clo[F] + 1];
            ++losS[cup[F] + 1];
        }
        for (int k = 0; k < nagg; ++k)
        {
            own[k + 1] += own[k];
            losS[k + 1] += losS[k];
        }
        {
            std::vector<int> pos(losS.begin(), losS.end() - 1);
            for (int F = 0; F < nfc; ++F) los[pos[cup[F]]++] = F;
        }
        HostLayout H;
        const double tl = wall_now();
        AMG_TRY(build_layout(nagg, nfc, clo.data(), cup.data(), own.data(), los.data(),
                             losS.data(), false, H));
        tLayout += wall_now() - tl;
        d->lv.emplace_back();
        AmgLevel& C = d->lv.back();
        C.n = nagg;
        C.nf = nfc;
        C.hLow = clo;
        C.hUpp = cup;
        C.nnzp = H.nnzp;
        int* sliceOff = nullptr;
        int* col = nullptr;
        float* val = nullptr;
        AMG_TRY(amg_upload(c, d, &sliceOff, H.sliceOff));
        AMG_TRY(amg_upload(c, d, &col, H.col));
        AMG_TRY(amg_upload(c, d, &C.eface, H.eface));
        AMG_TRY(amg_alloc(c, d, &val, (size_t)std::max(H.nnzp, 1LL)));
        C.A.n = nagg;
        C.A.nslices = H.nslices;
        C.A.sliceOff = sliceOff;
        C.A.col = col;
        C.A.val = val;
        C.A.val64 = nullptr;
        C.A.col16 = nullptr;
        C.A.ellW = H.uniformW;
        AMG_TRY(amg_alloc(c, d, &C.diag32, nagg));
        AMG_TRY(amg_alloc(c, d, &C.rD32, nagg));
        AMG_TRY(amg_alloc(c, d, &C.diag64, nagg));
        AMG_TRY(amg_alloc(c, d, &C.upper64, nfc));
        AMG_TRY(amg_alloc(c, d, &C.b, nagg));
        AMG_TRY(amg_alloc(c, d, &C.x0, nagg));
        AMG_TRY(amg_alloc(c, d, &C.x1, nagg));
        AMG_TRY(amg_alloc(c, d, &C.w, nagg));
        AMG_TRY(amg_alloc(c, d, &C.r, nagg));
        // the coarse level's coefficients on the host (the same Galerkin sums
        // the device forms for every solve), for the next aggregation
        {
            std::vector<double> cd(nagg, 0.0), cu(nfc, 0.0);
            for (int k = 0; k < nagg; ++k)
            {
                for (int q = aggStart[k]; q < aggStart[k + 1]; ++q) cd[k] += hd[aggRows[q]];
                for (int q = intStart[k]; q < intStart[k + 1]; ++q) cd[k] += 2.0 * hu[intList[q]];
            }
            for (int F = 0; F < nfc; ++F)
                for (int q = cfStart[F]; q < cfStart[F + 1]; ++q) cu[F] += hu[cfList[q]];
            hd.swap(cd);
            hu.swap(cu);
        }
        lo.swap(clo);
        up.swap(cup);
        cur = (int)d->lv.size() - 1;
        if (nagg * 10 > nl * 9) break;   // coarsening stalled
    }
    AmgLevel& Z = d->lv.back();
    if (d->lv.size() < 2 || Z.n > AMG_MAX_COARSEST)
    {
        amg_release(c);
        return fail(CF_ERR_UNSUPPORTED,
                    "GAMG: the mesh does not coarsen to at most 128 cells (disconnected or "
                    "too few faces)");
    }
    AMG_TRY(amg_alloc(c, d, &d->scale, 1));
    AMG_TRY(amg_alloc(c, d, &d->coarseInv, (size_t)Z.n * Z.n));
    AMG_CUDA(cudaStreamSynchronize(c->stream));
    if (profile)
    {
        std::printf("    GAMG hierarchy: %d levels (", (int)d->lv.size());
        for (size_t l = 0; l < d->lv.size(); ++l)
            std::printf("%s%d", l ? " / " : "", d->lv[l].n);
        std::printf(" cells) built in %.1f ms: aggregation %.1f, coarse faces %.1f, "
                    "layouts %.1f, rest (copies, uploads) %.1f\n",
                    1e3 * (wall_now() - t0), 1e3 * tAgg, 1e3 * tCoarse, 1e3 * tLayout,
                    1e3 * (wall_now() - t0 - tAgg - tCoarse - tLayout));
    }
    return CF_OK;
}

// Coefficients of every coarse level from the staged operator of level 0
// (diag64, or diag64 - u when deflating; the caller's upper).
int amg_stage(cf_context* c, int deflate, float scaleCorrection)
{
    AmgData* d = static_cast<AmgData*>(c->amg);
    if (!d) return fail(CF_ERR_INVALID_ARG, "GAMG hierarchy not built");
    cudaStream_t s = c->stream;
    d->hostScale = scaleCorrection;
    AMG_CUDA(cudaMemcpyAsync(d->scale, &d->hostScale, sizeof(float), cudaMemcpyHostToDevice, s));
    for (size_t l = 0; l + 1 < d->lv.size(); ++l)
    {
        AmgLevel& F = d->lv[l];
        AmgLevel& C = d->lv[l + 1];
        const double* upper = l == 0 ? c->d_upper : F.upper64;
        const double* diag = l == 0 ? c->d_diag64 : F.diag64;
        ka_coarse_upper<<<grid_n(c, (const void*)ka_coarse_upper, C.nf), NT, 0, s>>>(
            C.nf, F.cfStart, F.cfList, upper, C.upper64);
        AMG_LAUNCH();
        ka_coarse_diag<<<grid_n(c, (const void*)ka_coarse_diag, C.n), NT, 0, s>>>(
            C.n, F.aggStart, F.aggRows, F.intStart, F.intList, diag, c->d_u,
            (l == 0 && deflate) ? 1 : 0, upper, C.diag64, C.diag32, C.rD32);
        AMG_LAUNCH();
        ka_stage_vals<<<grid_n(c, (const void*)ka_stage_vals, C.nnzp), NT, 0, s>>>(
            C.nnzp, C.eface, C.upper64, const_cast<float*>(C.A.val));
        AMG_LAUNCH();
    }
    AmgLevel& Z = d->lv.back();
    const int smem = (Z.n * Z.n + Z.n) * (int)sizeof(double);
    // the attribute is the function's, shared by every context of the
    // process: always the same value (the largest coarsest level, 128
    // cells), so concurrent solves on other threads never lower it under a
    // launch that needs more
    constexpr int kMaxCoarse = 128;
    static_assert((kMaxCoarse * kMaxCoarse + kMaxCoarse) * sizeof(double) <= 227 * 1024,
                  "coarsest inverse must fit one CTA's shared memory");
    if (Z.n > kMaxCoarse) return fail(CF_ERR_UNSUPPORTED, "GAMG coarsest level above 128 cells");
    AMG_CUDA(cudaFuncSetAttribute(ka_coarse_invert, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (kMaxCoarse * kMaxCoarse + kMaxCoarse) * (int)sizeof(double)));
    ka_coarse_invert<<<1, AMG_INV_THREADS, smem, s>>>(Z.n, Z.A.sliceOff, Z.A.col, Z.eface,
                                                      Z.upper64, Z.diag64, deflate ? 1 : 0,
                                                      d->coarseInv);
    AMG_LAUNCH();
    return CF_OK;
}

// One inner PCG iteration with the V-cycle: z = M r, then the p-update SpMV
// and the update of metalFoamBackend::pcg (.C:676-715).
int launch_amg_body(cf_context* c, int degree, cudaGraphConditionalHandle h, int useCond,
                    int* kernels)
{
    AmgData* d = static_cast<AmgData*>(c->amg);
    if (!d || d->lv.size() < 2) return fail(CF_ERR_INVALID_ARG, "GAMG hierarchy not built");
    const long long l0 = c->launches;
    const DevSell A = sell_of(c);
    const PcgBufs B = pcg_bufs(c);
    cudaStream_t s = c->stream;
    float* Z[2] = {B.Z0, B.Z1};
    // level 0 pre-smoothing: w0 = c1 rD r is in W0 (formed by the update)
    const float* xa = B.W0;
    int zi = 0;
    for (int j = 1; j < degree; ++j)
    {
        auto fn = k_cheb_step<false, MW>;
        fn<<<rows_grid(c->n), NT, 0, s>>>(A, B, xa, j == 1 ? B.W0 : B.W1, B.W1, Z[zi], j, c->d_st,
                                          c->d_part);
        AMG_LAUNCH();
        xa = Z[zi];
        zi ^= 1;
    }
    float* x0 = const_cast<float*>(xa);
    // coarse-grid correction (the residual in Q, free until the p-update SpMV)
    ka_resid<MW><<<grid_for(c, (const void*)ka_resid<MW>, c->n), NT, 0, s>>>(
        A, B.diag, B.rA, x0, B.Q, c->d_st);
    AMG_LAUNCH();
    const AmgLevel& L0 = d->lv[0];
    float* xc = nullptr;
    // coarse levels smooth with degree 2: their Galerkin rows are wide, and
    // one step less there costs fewer iterations than it saves
    AMG_TRY(vcycle_coarse(c, d, 1, degree > AMG_COARSE_DEGREE ? AMG_COARSE_DEGREE : degree, B.Q,
                          &xc));
    // level 0 post-smoothing from x + a P x'; the last step forms z.r and beta
    float* xin = x0;
    float* xout = (x0 == Z[0]) ? Z[1] : Z[0];
    ka_step<MW, true><<<grid_for(c, (const void*)ka_step<MW, true>, c->n), NT, 0, s>>>(
        A, B.diag, B.rD, B.rA, xin, L0.agg, xc, d->scale, B.W1, xout, c->d_chebC, 0, c->d_st);
    AMG_LAUNCH();
    std::swap(xin, xout);
    for (int j = 1; j < degree; ++j)
    {
        if (j == degree - 1)
        {
            auto fn = k_cheb_step<true, MW>;
            fn<<<grid_for(c, (const void*)fn, c->n), NT, 0, s>>>(A, B, xin, B.W1, B.W1, xout, j,
                                                                c->d_st, c->d_part);
        }
        else
        {
            auto fn = k_cheb_step<false, MW>;
            fn<<<rows_grid(c->n), NT, 0, s>>>(A, B, xin, B.W1, B.W1, xout, j, c->d_st, c->d_part);
        }
        AMG_LAUNCH();
        std::swap(xin, xout);
    }
    const float* z = xin;
    {
        auto fn = k_pcg_p_spmv<MW>;
        fn<<<grid_for(c, (const void*)fn, c->n), NT, 0, s>>>(A, B, z, c->d_st, c->d_part);
        AMG_LAUNCH();
    }
    {
        auto fn = k_pcg_update<true>;
        fn<<<grid_for(c, (const void*)fn, c->n), NT, 0, s>>>(B, c->d_st, c->d_part, h, useCond);
        AMG_LAUNCH();
    }
    if (kernels) *kernels = (int)(c->launches - l0);
    return CF_OK;
}

}  // namespace cf

extern "C" int cf_gamg_levels(cf_context* c, int32_t* cells, int32_t capacity, int32_t* levels)
{
    if (!c || !levels || (capacity > 0 && !cells))
        return fail(CF_ERR_INVALID_ARG, "NULL argument");
    const int L = amg_levels(c);
    *levels = L;
    for (int l = 0; l < L && l < capacity; ++l) cells[l] = amg_level_cells(c, l);
    return CF_OK;
}

extern "C" int cf_gamg_export(cf_context* c, int32_t level, int32_t* nFaces, int32_t* agg,
                              double* diag, double* upper, int32_t* lowerAddr,
                              int32_t* upperAddr)
{
    if (!c || !nFaces) return fail(CF_ERR_INVALID_ARG, "NULL argument");
    AmgData* d = static_cast<AmgData*>(c->amg);
    if (!d || level < 1 || level >= (int)d->lv.size())
        return fail(CF_ERR_INVALID_ARG, "no such GAMG level (run a GAMG solve first)");
    const AmgLevel& F = d->lv[level - 1];
    const AmgLevel& L = d->lv[level];
    *nFaces = L.nf;
    if (agg)
    {
        if (level == 1)
            for (int r = 0; r < F.n; ++r) agg[c->perm[r]] = F.hAgg[r];
        else
            std::copy(F.hAgg.begin(), F.hAgg.end(), agg);
    }
    if (lowerAddr) std::copy(L.hLow.begin(), L.hLow.end(), lowerAddr);
    if (upperAddr) std::copy(L.hUpp.begin(), L.hUpp.end(), upperAddr);
    cudaError_t e = cudaSuccess;
    if (diag && e == cudaSuccess)
        e = cudaMemcpyAsync(diag, L.diag64, sizeof(double) * L.n, cudaMemcpyDeviceToHost, c->stream);
    if (upper && L.nf > 0 && e == cudaSuccess)
        e = cudaMemcpyAsync(upper, L.upper64, sizeof(double) * L.nf, cudaMemcpyDeviceToHost,
                            c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return fail(CF_ERR_CUDA, std::string("cf_gamg_export: ") + cudaGetErrorString(e));
    return CF_OK;
}
