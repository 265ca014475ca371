// cf_tune.cu -- launch-shape variants of the SpMV-carrying FP32 kernels and
// the autotuner that picks among them.
//
// A variant is (layout, rows per warp, block size):
//   SELL32 / 32 rows per warp: the SELL-32 copy, one row per thread -- the
//     kernels of cf_kernels.cuh at 256 threads, here at 128 or 512;
//   LDU / G lanes per row (rows per warp = 32 / G): the reference's own
//     addressing read directly, as ldu_spmv_dotw does
//     (metalFoamKernels.metal:64-109): the ownerStartAddr range of the row's
//     cell gives its faces f with upperAddr[f] / upper[f], the
//     losortStartAddr range gives losortAddr slots -> faces f with
//     lowerAddr[f] / lower[f].  Cells are relabelled to the internal order
//     once (uppI / lowI), the faces keep the caller's numbering.
// With G > 1 the lanes of a row load entries and form products side by
// side, then every lane adds the products in entry order (a shuffle per
// entry), so each row of A x is bit-identical to the one-thread-per-row
// result and to the reference kernel's sequential loop.
#include "cudafoam.h"
#include "cf_host.hpp"

#include <algorithm>
#include <string>
#include <type_traits>
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

namespace {

template <int V>
using IC = std::integral_constant<int, V>;

// ------------------------------------------------------------ reductions

template <int NR, int BS>
__device__ __forceinline__ void block_sum_bs(double (&v)[NR])
{
    __shared__ double sh[NR][BS / 32];
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
            double t = lane < BS / 32 ? sh[r][lane] : 0.0;
            v[r] = warp_sum(t);
        }
    }
}

// grid_sum of cf_kernels.cuh for BS-thread blocks (last-block-done fold)
template <int NR, int BS>
__device__ __forceinline__ bool grid_sum_bs(double (&v)[NR], double* part, unsigned int* ticket)
{
    __shared__ bool amLast;
    block_sum_bs<NR, BS>(v);
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
    for (int i = threadIdx.x; i < (int)gridDim.x; i += BS)
    {
#pragma unroll
        for (int r = 0; r < NR; ++r) acc[r] += __ldcg(part + r * gridDim.x + i);
    }
    block_sum_bs<NR, BS>(acc);
    if (threadIdx.x == 0)
    {
#pragma unroll
        for (int r = 0; r < NR; ++r) v[r] = acc[r];
        *ticket = 0u;
    }
    return true;
}

// ------------------------------------------------------------ row operators

struct SellOp
{
    DevSell A;
};

struct LduOp
{
    const int* cell;    // internal row -> caller's cell
    const int* own;     // ownerStartAddr (caller's cells)
    const int* losS;    // losortStartAddr
    const int* los;     // losortAddr
    const int* uppI;    // internal row of upperAddr[f]
    const int* lowI;    // internal row of lowerAddr[f]
    const float* up32;  // owner-side coefficient of face f
    const float* lo32;  // neighbour-side coefficient of face f
};

// acc + the off-diagonal products of row r in stored order (G must be 1)
template <int G, class XF>
__device__ __forceinline__ float op_row(const SellOp& o, int r, bool, float acc, XF xf, int)
{
    static_assert(G == 1, "the SELL-32 layout is read one row per thread");
    return row_f32<MAXW_UNROLL>(o.A, r, acc, xf);
}

// acc + the off-diagonal products of row r: owner-side faces (ascending f),
// then neighbour-side faces (losort order).  With G > 1 every lane of the
// row's group returns the same value; all 32 lanes of the warp must call it
// (rows past the end pass valid = false).
template <int G, class XF>
__device__ __forceinline__ float op_row(const LduOp& o, int r, bool valid, float acc, XF xf,
                                        int lane)
{
    int f0 = 0, nOwn = 0, q0 = 0, len = 0;
    if (valid)
    {
        const int cell = __ldg(o.cell + r);
        f0 = __ldg(o.own + cell);
        nOwn = __ldg(o.own + cell + 1) - f0;
        q0 = __ldg(o.losS + cell);
        len = nOwn + (__ldg(o.losS + cell + 1) - q0);
    }
    if (G == 1)
    {
        for (int k = 0; k < nOwn; ++k)
        {
            const int f = f0 + k;
            acc = __fadd_rn(acc, __fmul_rn(__ldg(o.up32 + f), xf(__ldg(o.uppI + f))));
        }
        for (int k = 0; k < len - nOwn; ++k)
        {
            const int f = __ldg(o.los + q0 + k);
            acc = __fadd_rn(acc, __fmul_rn(__ldg(o.lo32 + f), xf(__ldg(o.lowI + f))));
        }
        return acc;
    }
    // a trip count uniform over the warp keeps every shuffle converged
    const int wlen = __reduce_max_sync(0xffffffffu, len);
    for (int base = 0; base < wlen; base += G)
    {
        const int k = base + lane;
        float p = 0.0f;
        if (k < len)
        {
            int f, col;
            float v;
            if (k < nOwn)
            {
                f = f0 + k;
                v = __ldg(o.up32 + f);
                col = __ldg(o.uppI + f);
            }
            else
            {
                f = __ldg(o.los + q0 + (k - nOwn));
                v = __ldg(o.lo32 + f);
                col = __ldg(o.lowI + f);
            }
            p = __fmul_rn(v, xf(col));
        }
#pragma unroll
        for (int t = 0; t < G; ++t)
        {
            const float pt = __shfl_sync(0xffffffffu, p, t, G);
            if (base + t < len) acc = __fadd_rn(acc, pt);
        }
    }
    return acc;
}

// Rows of a launch: group g (G lanes) of the grid takes rows g, g + groups,
// ...; the loop bound is tested on the first row of the warp, so the loop
// is warp-uniform (rows past n arrive with valid = false).
#define CFT_ROWS(row, valid, n)                                                            \
    for (int row##_w = (int)((blockIdx.x * BS + (threadIdx.x & ~31u)) / G); row##_w < (n); \
         row##_w += (int)(gridDim.x * (BS / G)))                                           \
        for (int row = row##_w + (int)((threadIdx.x & 31u) / G), row##_1 = 1; row##_1;     \
             row##_1 = 0)                                                                  \
            for (bool valid = row < (n); row##_1; row##_1 = 0)

// ------------------------------------------------------------ kernels

template <class Op, int G, int BS>
__global__ void __launch_bounds__(BS) kt_spmv32(Op op, int n, const float* __restrict__ diag,
                                                const float* __restrict__ x,
                                                const float* __restrict__ w,
                                                float* __restrict__ y, double* out,
                                                unsigned int* ticket, double* part)
{
    const int lane = threadIdx.x & (G - 1);
    double acc[1] = {0.0};
    CFT_ROWS(row, valid, n)
    {
        if (G == 1 && !valid) continue;
        float v = valid ? __fmul_rn(diag[row], x[row]) : 0.0f;
        v = op_row<G>(op, row, valid, v, [&](int c) { return __ldg(x + c); }, lane);
        if (valid && lane == 0)
        {
            y[row] = v;
            if (w) acc[0] += (double)w[row] * (double)v;
        }
    }
    if (grid_sum_bs<1, BS>(acc, part, ticket) && threadIdx.x == 0) *out = acc[0];
}

// k_cheb_step in any launch shape
template <bool LAST, class Op, int G, int BS>
__global__ void __launch_bounds__(BS) kt_cheb_step(Op op, int n, PcgBufs B, const float* zin,
                                                   const float* win, float* wout, float* zout,
                                                   int j, InnerState* st, double* part)
{
    if (st->done) return;
    const int lane = threadIdx.x & (G - 1);
    const float c2 = B.chebC[2 * j - 1];
    const float c3 = B.chebC[2 * j];
    double acc[1] = {0.0};
    CFT_ROWS(row, valid, n)
    {
        if (G == 1 && !valid) continue;
        const float zr = valid ? zin[row] : 0.0f;
        float v = valid ? __fmul_rn(B.diag[row], zr) : 0.0f;
        v = op_row<G>(op, row, valid, v, [&](int c) { return __ldg(zin + c); }, lane);
        if (valid && lane == 0)
        {
            const float r = B.rA[row];
            const float wn = __fadd_rn(__fmul_rn(c2, win[row]),
                                       __fmul_rn(__fmul_rn(c3, B.rD[row]), __fsub_rn(r, v)));
            const float zn = __fadd_rn(zr, wn);
            wout[row] = wn;
            zout[row] = zn;
            if (LAST) acc[0] += (double)zn * (double)r;
        }
    }
    if (LAST)
    {
        if (grid_sum_bs<1, BS>(acc, part, &st->ticket) && threadIdx.x == 0)
        {
            st->wArAold = st->wArA;
            st->wArA = acc[0];
            st->beta = (st->it == 0) ? 0.0 : st->wArA / st->wArAold;
        }
    }
}

// k_pcg_p_spmv in any launch shape
template <class Op, int G, int BS>
__global__ void __launch_bounds__(BS) kt_pcg_p_spmv(Op op, int n, PcgBufs B, const float* wA,
                                                    InnerState* st, double* part)
{
    if (st->done) return;
    const int lane = threadIdx.x & (G - 1);
    const int par = st->it & 1;
    const float* __restrict__ Pold = B.P + (size_t)(par ^ 1) * n;
    float* __restrict__ Pn = B.P + (size_t)par * n;
    const float beta = (float)st->beta;
    auto pf = [&](int c) { return __fadd_rn(__ldg(wA + c), __fmul_rn(beta, __ldg(Pold + c))); };
    double acc[1] = {0.0};
    CFT_ROWS(row, valid, n)
    {
        if (G == 1 && !valid) continue;
        const float pr = valid ? pf(row) : 0.0f;
        float y = valid ? __fmul_rn(B.diag[row], pr) : 0.0f;
        y = op_row<G>(op, row, valid, y, pf, lane);
        if (valid && lane == 0)
        {
            Pn[row] = pr;
            B.Q[row] = y;
            acc[0] += (double)pr * (double)y;
        }
    }
    if (grid_sum_bs<1, BS>(acc, part, &st->ticket) && threadIdx.x == 0)
    {
        st->wApA = acc[0];
        st->alpha = st->wArA / st->wApA;
    }
}

// k_bicg_ab in any launch shape
template <class Op, int G, int BS>
__global__ void __launch_bounds__(BS) kt_bicg_ab(Op op, int n, BicgBufs B, InnerState* st,
                                                 double* part)
{
    if (st->done) return;
    const int lane = threadIdx.x & (G - 1);
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
    CFT_ROWS(row, valid, n)
    {
        if (G == 1 && !valid) continue;
        const float p = valid ? pf(row) : 0.0f;
        const float y = valid ? __fmul_rn(B.rD[row], p) : 0.0f;
        float v = valid ? __fmul_rn(B.diag[row], y) : 0.0f;
        v = op_row<G>(op, row, valid, v, yf, lane);
        if (valid && lane == 0)
        {
            Pn[row] = p;
            B.yA[row] = y;
            An[row] = v;
            acc[0] += (double)B.rA0[row] * (double)v;
        }
    }
    if (grid_sum_bs<1, BS>(acc, part, &st->ticket) && threadIdx.x == 0)
    {
        st->rA0AyA = acc[0];
        st->alpha = st->rA0rA / st->rA0AyA;
    }
}

// k_bicg_cd in any launch shape
template <class Op, int G, int BS>
__global__ void __launch_bounds__(BS) kt_bicg_cd(Op op, int n, BicgBufs B, InnerState* st,
                                                 double* part, cudaGraphConditionalHandle h,
                                                 int useCond)
{
    if (st->done) return;
    const int lane = threadIdx.x & (G - 1);
    const int par = st->it & 1;
    const float* __restrict__ An = B.AyA + (size_t)par * n;
    const float alpha = (float)st->alpha;
    auto zf = [&](int c) {
        return __fmul_rn(__ldg(B.rD + c), __fsub_rn(__ldg(B.rA + c), __fmul_rn(alpha, __ldg(An + c))));
    };
    double acc[3] = {0.0, 0.0, 0.0};
    CFT_ROWS(row, valid, n)
    {
        if (G == 1 && !valid) continue;
        const float sv = valid ? __fsub_rn(B.rA[row], __fmul_rn(alpha, An[row])) : 0.0f;
        const float z = valid ? __fmul_rn(B.rD[row], sv) : 0.0f;
        float t = valid ? __fmul_rn(B.diag[row], z) : 0.0f;
        t = op_row<G>(op, row, valid, t, zf, lane);
        if (valid && lane == 0)
        {
            B.sA[row] = sv;
            B.zA[row] = z;
            B.tA[row] = t;
            acc[0] += (double)fabsf(sv);
            acc[1] += (double)sv * (double)t;
            acc[2] += (double)t * (double)t;
        }
    }
    if (grid_sum_bs<3, BS>(acc, part, &st->ticket) && threadIdx.x == 0)
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

// R-component SpMV reading each SELL entry once (the multi-RHS inner
// product of cf_solve_multi), timed by the autotuner for the RHS tile
template <int R>
__global__ void __launch_bounds__(NT) kt_spmv_multi(DevSell A, const float* __restrict__ diag,
                                                    const float* __restrict__ x,
                                                    float* __restrict__ y, long long ld)
{
    CF_ROWS(row, A.n)
    {
        const int sl = row >> 5;
        const int b0 = __ldg(A.sliceOff + sl);
        const int w = (__ldg(A.sliceOff + sl + 1) - b0) >> 5;
        const int base = b0 + (row & 31);
        const float dg = diag[row];
        float acc[R];
#pragma unroll
        for (int r = 0; r < R; ++r) acc[r] = __fmul_rn(dg, x[r * ld + row]);
        for (int k = 0; k < w; ++k)
        {
            const int c = __ldcs(A.col + base + SLICE * k);
            if (c == -1) continue;
            const float v = __ldcs(A.val + base + SLICE * k);
            const int ci = col_index(c);
#pragma unroll
            for (int r = 0; r < R; ++r) acc[r] = __fadd_rn(acc[r], __fmul_rn(v, __ldg(x + r * ld + ci)));
        }
#pragma unroll
        for (int r = 0; r < R; ++r) y[r * ld + row] = acc[r];
    }
}

__global__ void kt_stage_face32(int nf, const double* __restrict__ up, const double* __restrict__ lo,
                                int sym32, float* __restrict__ up32, float* __restrict__ lo32)
{
    for (int f = blockIdx.x * NT + threadIdx.x; f < nf; f += gridDim.x * NT)
    {
        up32[f] = (float)up[f];
        lo32[f] = (float)(sym32 ? up[f] : lo[f]);
    }
}

__global__ void kt_fill(long long count, float* __restrict__ x)
{
    for (long long i = (long long)blockIdx.x * NT + threadIdx.x; i < count;
         i += (long long)gridDim.x * NT)
        x[i] = 1.0f + 0.25f * (float)(i % 7);
}

// ------------------------------------------------------------ host

int launched(cf_context* c)
{
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(CF_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    c->launches++;
    return CF_OK;
}

// blocks for a variant launch: resident capacity of the kernel at BS
// threads, or one group per row if fewer
int grid_v(cf_context* c, const void* fn, int n, int G, int BS)
{
    int occ = 0;
    auto it = c->occ.find(fn);
    if (it == c->occ.end())
    {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, BS, 0) != cudaSuccess) occ = 1;
        occ = std::max(1, std::min(occ, c->maxCtasPerSM));
        c->occ[fn] = occ;
    }
    else
    {
        occ = it->second;
    }
    const long long groupsPerBlock = BS / G;
    const long long need = ((long long)n + groupsPerBlock - 1) / groupsPerBlock;
    return (int)std::max(1LL, std::min((long long)c->numSMs * occ, need));
}

LduOp ldu_of(const cf_context* c)
{
    LduOp o;
    o.cell = c->d_perm;
    o.own = c->d_own;
    o.losS = c->d_losS;
    o.los = c->d_los;
    o.uppI = c->d_uppI;
    o.lowI = c->d_lowI;
    o.up32 = c->d_face32;
    o.lo32 = c->d_face32 + c->nf;
    return o;
}

template <class T>
int talloc(cf_context* c, T** p, size_t count)
{
    *p = nullptr;
    const cudaError_t e = cudaMalloc((void**)p, std::max<size_t>(count, 1) * sizeof(T));
    if (e != cudaSuccess) return fail(CF_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    c->topoAllocs.push_back((void*)*p);
    return CF_OK;
}

// The reference's addressing on the device, relabelled columns and FP32
// face coefficients (built from the uploaded face arrays on first use).
int ensure_ldu(cf_context* c)
{
    if (c->lduReady) return CF_OK;
    if (!c->hasTopo) return fail(CF_ERR_NO_TOPOLOGY, "cf_set_topology has not been called");
    const int n = c->n, nf = c->nf;
    std::vector<int32_t> low(nf), upp(nf);
    CF_CUDA(cudaMemcpy(low.data(), c->d_low, sizeof(int32_t) * nf, cudaMemcpyDeviceToHost));
    CF_CUDA(cudaMemcpy(upp.data(), c->d_upp, sizeof(int32_t) * nf, cudaMemcpyDeviceToHost));
    // ownerStart / losortStart / losort of validated LDU addressing
    // (faces sorted by owner, losort stable in the face index)
    std::vector<int32_t> own(n + 1, 0), losS(n + 1, 0), los(nf), uppI(nf), lowI(nf), iperm(n);
    for (int32_t f = 0; f < nf; ++f)
    {
        own[low[f] + 1]++;
        losS[upp[f] + 1]++;
    }
    for (int32_t i = 0; i < n; ++i)
    {
        own[i + 1] += own[i];
        losS[i + 1] += losS[i];
    }
    std::vector<int32_t> pos(losS.begin(), losS.end() - 1);
    for (int32_t f = 0; f < nf; ++f) los[pos[upp[f]]++] = f;
    for (int32_t r = 0; r < n; ++r) iperm[c->perm[r]] = r;
    for (int32_t f = 0; f < nf; ++f)
    {
        uppI[f] = iperm[upp[f]];
        lowI[f] = iperm[low[f]];
    }
    CF_TRY(talloc(c, &c->d_own, n + 1));
    CF_TRY(talloc(c, &c->d_losS, n + 1));
    CF_TRY(talloc(c, &c->d_los, nf));
    CF_TRY(talloc(c, &c->d_uppI, nf));
    CF_TRY(talloc(c, &c->d_lowI, nf));
    CF_TRY(talloc(c, &c->d_face32, 2 * (size_t)nf));
    CF_CUDA(cudaMemcpy(c->d_own, own.data(), sizeof(int32_t) * (n + 1), cudaMemcpyHostToDevice));
    CF_CUDA(cudaMemcpy(c->d_losS, losS.data(), sizeof(int32_t) * (n + 1), cudaMemcpyHostToDevice));
    CF_CUDA(cudaMemcpy(c->d_los, los.data(), sizeof(int32_t) * nf, cudaMemcpyHostToDevice));
    CF_CUDA(cudaMemcpy(c->d_uppI, uppI.data(), sizeof(int32_t) * nf, cudaMemcpyHostToDevice));
    CF_CUDA(cudaMemcpy(c->d_lowI, lowI.data(), sizeof(int32_t) * nf, cudaMemcpyHostToDevice));
    c->lduReady = true;
    if (c->hasCoeffs)
    {
        const double* up = c->d_upper;
        const double* lo = c->hasLower ? c->d_lower : c->d_upper;
        if (c->transposed) std::swap(up, lo);
        CF_TRY(stage_face32(c, up, lo, c->val32Sym));
    }
    return CF_OK;
}

bool valid_config(const cf_spmv_config& k)
{
    if (k.indexBits != 16 && k.indexBits != 32) return false;
    if (k.blockSize != 128 && k.blockSize != 256 && k.blockSize != 512) return false;
    if (k.rhsTile < 0 || k.rhsTile > 4) return false;
    if (k.layout == CF_LAYOUT_SELL32) return k.rowsPerWarp == 32;
    if (k.layout == CF_LAYOUT_LDU)
        return k.rowsPerWarp == 32 || k.rowsPerWarp == 8 || k.rowsPerWarp == 4 ||
               k.rowsPerWarp == 1;
    return false;
}

// Calls f(op, IC<G>, IC<BS>) for the context's variant.
template <class F>
int dispatch(cf_context* c, F&& f)
{
    if (c->cfgLayout == CF_LAYOUT_SELL32)
    {
        const SellOp op{sell_of(c)};
        switch (c->cfgBlockSize)
        {
            case 128: return f(op, IC<1>{}, IC<128>{});
            case 256: return f(op, IC<1>{}, IC<256>{});
            case 512: return f(op, IC<1>{}, IC<512>{});
            default: break;
        }
    }
    else if (c->cfgLayout == CF_LAYOUT_LDU)
    {
        CF_TRY(ensure_ldu(c));
        const LduOp op = ldu_of(c);
        const int G = 32 / c->cfgRowsPerWarp;
        switch (G * 10000 + c->cfgBlockSize)
        {
            case 10128: return f(op, IC<1>{}, IC<128>{});
            case 10256: return f(op, IC<1>{}, IC<256>{});
            case 10512: return f(op, IC<1>{}, IC<512>{});
            case 40128: return f(op, IC<4>{}, IC<128>{});
            case 40256: return f(op, IC<4>{}, IC<256>{});
            case 40512: return f(op, IC<4>{}, IC<512>{});
            case 80128: return f(op, IC<8>{}, IC<128>{});
            case 80256: return f(op, IC<8>{}, IC<256>{});
            case 80512: return f(op, IC<8>{}, IC<512>{});
            case 320128: return f(op, IC<32>{}, IC<128>{});
            case 320256: return f(op, IC<32>{}, IC<256>{});
            case 320512: return f(op, IC<32>{}, IC<512>{});
            default: break;
        }
    }
    return fail(CF_ERR_INVALID_ARG, "invalid SpMV launch configuration");
}

cf_spmv_config config_of(const cf_context* c)
{
    cf_spmv_config k;
    k.layout = c->cfgLayout;
    k.rowsPerWarp = c->cfgRowsPerWarp;
    k.blockSize = c->cfgBlockSize;
    k.rhsTile = c->cfgRhsTile;
    k.indexBits = c->cfgIndexBits;
    return k;
}

void apply_config(cf_context* c, const cf_spmv_config& k)
{
    const bool shapeChanged = k.layout != c->cfgLayout || k.rowsPerWarp != c->cfgRowsPerWarp ||
                              k.blockSize != c->cfgBlockSize || k.indexBits != c->cfgIndexBits;
    c->cfgLayout = k.layout;
    c->cfgRowsPerWarp = k.rowsPerWarp;
    c->cfgBlockSize = k.blockSize;
    c->cfgRhsTile = k.rhsTile;
    c->cfgIndexBits = k.indexBits;
    if (shapeChanged)
    {
        // captured inner loops hold the previous shape's kernels
        for (auto& kv : c->graphs) cudaGraphExecDestroy(kv.second);
        c->graphs.clear();
    }
}

}  // namespace

namespace cf {

bool spmv_default(const cf_context* c)
{
    return c->cfgLayout == CF_LAYOUT_SELL32 && c->cfgBlockSize == NT;
}

int stage_face32(cf_context* c, const double* up, const double* lo, int sym32)
{
    const int g = grid_for(c, (const void*)kt_stage_face32, c->nf);
    kt_stage_face32<<<g, NT, 0, c->stream>>>(c->nf, up, lo, sym32, c->d_face32,
                                             c->d_face32 + c->nf);
    return launched(c);
}

int launch_cheb_step_v(cf_context* c, bool last, const PcgBufs& B, const float* zin,
                       const float* win, float* wout, float* zout, int j)
{
    return dispatch(c, [&](const auto& op, auto g, auto b) -> int {
        using Op = std::decay_t<decltype(op)>;
        constexpr int G = decltype(g)::value;
        constexpr int BS = decltype(b)::value;
        if (last)
        {
            auto fn = kt_cheb_step<true, Op, G, BS>;
            fn<<<grid_v(c, (const void*)fn, c->n, G, BS), BS, 0, c->stream>>>(
                op, c->n, B, zin, win, wout, zout, j, c->d_st, c->d_part);
        }
        else
        {
            auto fn = kt_cheb_step<false, Op, G, BS>;
            fn<<<grid_v(c, (const void*)fn, c->n, G, BS), BS, 0, c->stream>>>(
                op, c->n, B, zin, win, wout, zout, j, c->d_st, c->d_part);
        }
        return launched(c);
    });
}

int launch_pcg_p_spmv_v(cf_context* c, const PcgBufs& B, const float* wA)
{
    return dispatch(c, [&](const auto& op, auto g, auto b) -> int {
        using Op = std::decay_t<decltype(op)>;
        constexpr int G = decltype(g)::value;
        constexpr int BS = decltype(b)::value;
        auto fn = kt_pcg_p_spmv<Op, G, BS>;
        fn<<<grid_v(c, (const void*)fn, c->n, G, BS), BS, 0, c->stream>>>(op, c->n, B, wA,
                                                                           c->d_st, c->d_part);
        return launched(c);
    });
}

int launch_bicg_ab_v(cf_context* c, const BicgBufs& B)
{
    return dispatch(c, [&](const auto& op, auto g, auto b) -> int {
        using Op = std::decay_t<decltype(op)>;
        constexpr int G = decltype(g)::value;
        constexpr int BS = decltype(b)::value;
        auto fn = kt_bicg_ab<Op, G, BS>;
        fn<<<grid_v(c, (const void*)fn, c->n, G, BS), BS, 0, c->stream>>>(op, c->n, B, c->d_st,
                                                                           c->d_part);
        return launched(c);
    });
}

int launch_bicg_cd_v(cf_context* c, const BicgBufs& B, cudaGraphConditionalHandle h, int useCond)
{
    return dispatch(c, [&](const auto& op, auto g, auto b) -> int {
        using Op = std::decay_t<decltype(op)>;
        constexpr int G = decltype(g)::value;
        constexpr int BS = decltype(b)::value;
        auto fn = kt_bicg_cd<Op, G, BS>;
        fn<<<grid_v(c, (const void*)fn, c->n, G, BS), BS, 0, c->stream>>>(op, c->n, B, c->d_st,
                                                                           c->d_part, h, useCond);
        return launched(c);
    });
}

int launch_spmv32_v(cf_context* c, const float* diag, const float* x, const float* w, float* y,
                    double* out)
{
    return dispatch(c, [&](const auto& op, auto g, auto b) -> int {
        using Op = std::decay_t<decltype(op)>;
        constexpr int G = decltype(g)::value;
        constexpr int BS = decltype(b)::value;
        auto fn = kt_spmv32<Op, G, BS>;
        fn<<<grid_v(c, (const void*)fn, c->n, G, BS), BS, 0, c->stream>>>(
            op, c->n, diag, x, w, y, out, &c->d_drv->ticket, c->d_part);
        return launched(c);
    });
}

}  // namespace cf

// ------------------------------------------------------------------ C ABI

namespace {

int check_ctx(cf_context* c)
{
    if (!c) return fail(CF_ERR_INVALID_ARG, "context is NULL");
    const cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return fail(CF_ERR_CUDA, cudaGetErrorString(e));
    return CF_OK;
}

// FP32 SpMV + dot in the context's shape (the default shape runs k_spmv32)
int spmv_once(cf_context* c, const float* x, const float* w, float* y)
{
    if (spmv_default(c))
    {
        auto fn = k_spmv32<MAXW_UNROLL>;
        fn<<<grid_for(c, (const void*)fn, c->n), NT, 0, c->stream>>>(
            sell_of(c), c->d_diag32, x, w, y, c->d_scratch64, &c->d_drv->ticket, c->d_part);
        return launched(c);
    }
    return launch_spmv32_v(c, c->d_diag32, x, w, y, c->d_scratch64);
}

template <int R>
int multi_once(cf_context* c, const float* x, float* y)
{
    auto fn = kt_spmv_multi<R>;
    fn<<<grid_for(c, (const void*)fn, c->n), NT, 0, c->stream>>>(sell_of(c), c->d_diag32, x, y,
                                                                 (long long)c->n);
    return launched(c);
}

int multi_launch(cf_context* c, int R, const float* x, float* y)
{
    switch (R)
    {
        case 1: return multi_once<1>(c, x, y);
        case 2: return multi_once<2>(c, x, y);
        case 3: return multi_once<3>(c, x, y);
        default: return multi_once<4>(c, x, y);
    }
}

}  // namespace

extern "C" int cf_spmv_config_default(cf_spmv_config* k)
{
    if (!k) return fail(CF_ERR_INVALID_ARG, "config is NULL");
    k->layout = CF_LAYOUT_SELL32;
    k->rowsPerWarp = 32;
    k->blockSize = NT;
    k->rhsTile = 0;
    k->indexBits = 16;
    return CF_OK;
}

extern "C" int cf_get_spmv_config(cf_context* c, cf_spmv_config* k)
{
    if (!c || !k) return fail(CF_ERR_INVALID_ARG, "NULL argument");
    *k = config_of(c);
    return CF_OK;
}

extern "C" int cf_set_spmv_config(cf_context* c, const cf_spmv_config* k)
{
    CF_TRY(check_ctx(c));
    if (!k) return fail(CF_ERR_INVALID_ARG, "config is NULL");
    if (!valid_config(*k))
        return fail(CF_ERR_UNSUPPORTED,
                    "SpMV configuration not offered (layout SELL32: rowsPerWarp 32; layout LDU: "
                    "rowsPerWarp 32, 8, 4 or 1; blockSize 128, 256 or 512; rhsTile 0..4; "
                    "indexBits 16 or 32)");
    if (k->layout == CF_LAYOUT_LDU)
    {
        if (!c->hasTopo) return fail(CF_ERR_NO_TOPOLOGY, "cf_set_topology has not been called");
        CF_TRY(ensure_ldu(c));
    }
    apply_config(c, *k);
    return CF_OK;
}

extern "C" int cf_autotune(cf_context* c, int32_t reps, int32_t apply, cf_spmv_config* best,
                           cf_tune_entry* table, int32_t capacity, int32_t* count)
{
    CF_TRY(check_ctx(c));
    if (!c->hasTopo) return fail(CF_ERR_NO_TOPOLOGY, "cf_set_topology has not been called");
    if (!c->hasCoeffs) return fail(CF_ERR_NO_COEFFS, "cf_set_coeffs has not been called");
    if (!best || reps <= 0 || (capacity > 0 && !table))
        return fail(CF_ERR_INVALID_ARG, "bad arguments");
    CF_TRY(ensure_ldu(c));
    const cf_spmv_config saved = config_of(c);
    const int n = c->n;
    cudaStream_t s = c->stream;
    // operands: x in Z0, w in W0, y in W1 (finite, fixed values)
    const int g = grid_for(c, (const void*)kt_fill, n);
    kt_fill<<<g, NT, 0, s>>>(n, c->d_Z0);
    CF_TRY(launched(c));
    kt_fill<<<g, NT, 0, s>>>(n, c->d_W0);
    CF_TRY(launched(c));

    std::vector<cf_spmv_config> cand;
    for (int bits : {16, 32})
    {
        if (bits == 16 && !c->d_col16) continue;   // offsets do not fit: no compact stream
        for (int bs : {128, 256, 512})
            cand.push_back({CF_LAYOUT_SELL32, 32, bs, saved.rhsTile, bits});
    }
    for (int rpw : {32, 8, 4, 1})
        for (int bs : {128, 256, 512})
            cand.push_back({CF_LAYOUT_LDU, rpw, bs, saved.rhsTile, 32});
    int nt = 0;
    double bestMs = 1e300;
    cf_spmv_config win = saved;
    int rc = CF_OK;
    for (const cf_spmv_config& k : cand)
    {
        apply_config(c, k);
        rc = spmv_once(c, c->d_Z0, c->d_W0, c->d_W1);   // warm-up
        if (rc != CF_OK) break;
        cudaEventRecord(c->ev0, s);
        for (int i = 0; i < reps && rc == CF_OK; ++i) rc = spmv_once(c, c->d_Z0, c->d_W0, c->d_W1);
        cudaEventRecord(c->ev1, s);
        if (rc != CF_OK) break;
        if (cudaEventSynchronize(c->ev1) != cudaSuccess)
        {
            rc = fail(CF_ERR_CUDA, "cf_autotune: event synchronisation failed");
            break;
        }
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, c->ev0, c->ev1);
        const double per = (double)ms / reps;
        if (nt < capacity) table[nt] = {k, per};
        ++nt;
        if (per < bestMs)
        {
            bestMs = per;
            win = k;
        }
    }
    apply_config(c, saved);
    if (rc != CF_OK) return rc;

    // RHS tile of the fused multi-RHS form: least time per component of the
    // multi-component SpMV.  The concurrent form (rhsTile 0, whole solves
    // side by side) is kept: an SpMV timing cannot rank it against the fused
    // passes.
    if (saved.rhsTile == 0)
    {
        win.rhsTile = 0;
        *best = win;
        if (count) *count = nt;
        if (apply) apply_config(c, win);
        return CF_OK;
    }
    float* xm = nullptr;
    float* ym = nullptr;
    if (cudaMalloc((void**)&xm, sizeof(float) * 4 * (size_t)n) != cudaSuccess ||
        cudaMalloc((void**)&ym, sizeof(float) * 4 * (size_t)n) != cudaSuccess)
    {
        cudaGetLastError();
        cudaFree(xm);
        return fail(CF_ERR_CUDA, "cf_autotune: allocation of multi-RHS operands failed");
    }
    double bestPer = 1e300;
    int tile = 1;
    kt_fill<<<g, NT, 0, s>>>(4LL * n, xm);
    rc = launched(c);
    for (int R = 1; R <= 4 && rc == CF_OK; ++R)
    {
        rc = multi_launch(c, R, xm, ym);
        cudaEventRecord(c->ev0, s);
        for (int i = 0; i < reps && rc == CF_OK; ++i) rc = multi_launch(c, R, xm, ym);
        cudaEventRecord(c->ev1, s);
        if (rc != CF_OK) break;
        if (cudaEventSynchronize(c->ev1) != cudaSuccess)
        {
            rc = fail(CF_ERR_CUDA, "cf_autotune: event synchronisation failed");
            break;
        }
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, c->ev0, c->ev1);
        const double perComponent = (double)ms / reps / R;
        if (perComponent < bestPer)
        {
            bestPer = perComponent;
            tile = R;
        }
    }
    cudaFree(xm);
    cudaFree(ym);
    if (rc != CF_OK) return rc;
    win.rhsTile = tile;
    *best = win;
    if (count) *count = nt;
    if (apply) apply_config(c, win);
    return CF_OK;
}
