// cf_cluster.cu -- the inner PCG of a small mesh inside ONE thread-block
// cluster.
//
// A mesh of up to 16,384 cells fits one cluster of up to 16 CTAs x 1024
// threads, one row per thread: CTA k owns the rows [k RPC, (k + 1) RPC) (RPC
// the smallest power of two >= 32 that needs at most 16 CTAs) and keeps
// every work vector of its rows in its shared memory (rA, w, the
// Chebyshev z ping-pong, p ping-pong, q, and the three correction buffers
// of the minimum-residual iterate).  A column of another CTA is read from
// that CTA's shared memory (distributed shared memory, mapa + ld through the
// cluster window); the matrix stays in global memory on the read-only path
// (L1-resident after the first sweep).  Phases are separated by the
// hardware cluster barrier, and every reduction is: per-CTA sum -> one slot
// per CTA -> cluster barrier -> warp 0 of EVERY CTA folds the CTA sums in
// rank order, so all CTAs compute bit-identical scalars and run the same
// bookkeeping (inner_sync_point) on a private copy of the solver state: no
// broadcast, no global memory traffic inside the loop.
//
// Per row the arithmetic is row_f32's (same entries, same order, same
// rounding); the dot products fold per thread, per CTA and per cluster in
// an order of their own, so the scalars can differ from the graph path in
// the last bits (the tests compare convergence and iteration counts).
//
// The cluster path starts from the state k_inner_setup / k_pcg_init leave
// in global memory and ends by writing the solver state and the current and
// best corrections back, so the FP64 driver continues unchanged.
#include "cudafoam.h"
#include "cf_host.hpp"

#include <cooperative_groups.h>

#include <algorithm>
#include <string>

using namespace cf;
namespace cg = cooperative_groups;

namespace {

constexpr int CT = 1024;               // threads per CTA
constexpr int NVEC = 11;               // rA W0 W1 Z0 Z1 P0 P1 Q D0 D1 D2
constexpr int MW = MAXW_UNROLL;
enum { V_RA = 0, V_W0, V_W1, V_Z0, V_Z1, V_P0, V_P1, V_Q, V_D0 };

struct CArgs
{
    DevSell A;
    const float* diag;
    const float* rD;
    const float* chebC;
    const float* rA;          // global, after k_pcg_init
    const float* W0;
    InnerState* st;           // global state in / out
    float* D;                 // global corrections [3n]
    int n;
    int order;
    int shift;                // log2(RPC)
    int cs;                   // CTAs in the cluster
};

// one FP32 row of A x in row_f32's order, matrix entries through the
// read-only path (they are reused every phase)
template <class XF>
__device__ __forceinline__ float crow(const DevSell& A, int row, float acc, XF xf)
{
    const int s = row >> 5;
    const int b0 = A.ellW ? s * SLICE * A.ellW : __ldg(A.sliceOff + s);
    const int w = A.ellW ? A.ellW : (__ldg(A.sliceOff + s + 1) - b0) >> 5;
    const int base = b0 + (row & 31);
    if (w <= MW)
    {
        int c[MW];
        float v[MW];
#pragma unroll
        for (int k = 0; k < MW; ++k)
        {
            c[k] = -1;
            v[k] = 0.0f;
            if (k < w)
            {
                if (A.col16)
                {
                    const short o = __ldg(A.col16 + base + SLICE * k);
                    c[k] = o == COL16_PAD ? -1 : row + o;
                }
                else
                {
                    const int cc = __ldg(A.col + base + SLICE * k);
                    c[k] = cc == -1 ? -1 : col_index(cc);
                }
                v[k] = __ldg(A.val + base + SLICE * k);
            }
        }
        float x[MW];
#pragma unroll
        for (int k = 0; k < MW; ++k) x[k] = c[k] != -1 ? xf(c[k]) : 0.0f;
#pragma unroll
        for (int k = 0; k < MW; ++k)
            if (c[k] != -1) acc = __fadd_rn(acc, __fmul_rn(v[k], x[k]));
        return acc;
    }
    for (int k = 0; k < w; ++k)
    {
        int c;
        if (A.col16)
        {
            const short o = __ldg(A.col16 + base + SLICE * k);
            c = o == COL16_PAD ? -1 : row + o;
        }
        else
        {
            const int cc = __ldg(A.col + base + SLICE * k);
            c = cc == -1 ? -1 : col_index(cc);
        }
        if (c != -1) acc = __fadd_rn(acc, __fmul_rn(__ldg(A.val + base + SLICE * k), xf(c)));
    }
    return acc;
}

struct Shared
{
    double slot[2][4];        // this CTA's sums of the last two reductions
    double red[4][32];        // CTA-level reduction scratch
    double tot[4];            // cluster totals, broadcast inside the CTA
    InnerState S;             // this CTA's copy of the solver state
};

// Sum of NR values over the cluster; every thread of every CTA gets the
// totals (folded in rank order, identical in all CTAs).  Contains the
// cluster barrier that ends the phase.
template <int NR>
__device__ __forceinline__ void cluster_sum(double (&v)[NR], Shared& sh, int slot,
                                            const cg::cluster_group& cl, int cs)
{
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
#pragma unroll
    for (int r = 0; r < NR; ++r) v[r] = warp_sum(v[r]);
    if (lane == 0)
    {
#pragma unroll
        for (int r = 0; r < NR; ++r) sh.red[r][wid] = v[r];
    }
    __syncthreads();
    if (wid == 0)
    {
#pragma unroll
        for (int r = 0; r < NR; ++r)
        {
            const double t = warp_sum(lane < CT / 32 ? sh.red[r][lane] : 0.0);
            if (lane == 0) sh.slot[slot][r] = t;
        }
    }
    cl.sync();
    if (wid == 0)
    {
#pragma unroll
        for (int r = 0; r < NR; ++r)
        {
            double t = 0.0;
            if (lane < cs)
            {
                const Shared* rs = cl.map_shared_rank(&sh, (unsigned)lane);
                t = rs->slot[slot][r];
            }
            t = warp_sum(t);
            if (lane == 0) sh.tot[r] = t;
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < NR; ++r) v[r] = sh.tot[r];
}

template <bool CHEB>
__global__ void __launch_bounds__(CT, 1) kc_pcg(CArgs a)
{
    extern __shared__ float4 dyn[];
    float* vec = reinterpret_cast<float*>(dyn);
    __shared__ Shared sh;
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    const int rpc = 1 << a.shift;
    const int mask = rpc - 1;
    const int r0 = rank << a.shift;
    const int rows = max(0, min(rpc, a.n - r0));
    auto V = [&](int k) { return vec + (size_t)k * rpc; };
    // x[c] of vector k, from the owner CTA's shared memory
    auto X = [&](int k, int c) -> float {
        const int owner = c >> a.shift;
        const float* p = V(k) + (c & mask);
        if (owner == rank) return *p;
        return *cl.map_shared_rank(p, (unsigned)owner);
    };

    if (threadIdx.x == 0) sh.S = *a.st;
    for (int l = threadIdx.x; l < rows; l += CT)
    {
        V(V_RA)[l] = a.rA[r0 + l];
        V(V_W0)[l] = a.W0[r0 + l];
        V(V_D0)[l] = 0.0f;
        V(V_P0)[l] = 0.0f;
        V(V_P1)[l] = 0.0f;
    }
    __syncthreads();
    cl.sync();
    int slot = 0;
    InnerState& S = sh.S;
    const float c1 = CHEB ? __ldg(a.chebC) : 0.0f;
    while (!S.done)
    {
        if (CHEB)
        {
            for (int j = 1; j < a.order; ++j)
            {
                const int zin = (j == 1) ? V_W0 : (((j - 1) & 1) ? V_Z1 : V_Z0);
                const int win = (j == 1) ? V_W0 : V_W1;
                const int zout = (j & 1) ? V_Z1 : V_Z0;
                const float c2 = __ldg(a.chebC + 2 * j - 1);
                const float c3 = __ldg(a.chebC + 2 * j);
                const bool last = (j == a.order - 1);
                double acc[1] = {0.0};
                for (int l = threadIdx.x; l < rows; l += CT)
                {
                    const int row = r0 + l;
                    const float zr = V(zin)[l];
                    const float v = crow(a.A, row, __fmul_rn(__ldg(a.diag + row), zr),
                                         [&](int c) { return X(zin, c); });
                    const float r = V(V_RA)[l];
                    const float wn = __fadd_rn(__fmul_rn(c2, V(win)[l]),
                                               __fmul_rn(__fmul_rn(c3, __ldg(a.rD + row)),
                                                         __fsub_rn(r, v)));
                    const float zn = __fadd_rn(zr, wn);
                    V(V_W1)[l] = wn;
                    V(zout)[l] = zn;
                    if (last) acc[0] += (double)zn * (double)r;
                }
                if (last)
                {
                    cluster_sum<1>(acc, sh, slot, cl, a.cs);
                    slot ^= 1;
                    if (threadIdx.x == 0)
                    {
                        S.wArAold = S.wArA;
                        S.wArA = acc[0];
                        S.beta = (S.it == 0) ? 0.0 : S.wArA / S.wArAold;
                    }
                    __syncthreads();
                }
                else
                {
                    cl.sync();
                }
            }
        }
        // p-update fused into the SpMV gather, q = A p, p.q -> alpha
        {
            const int wA = CHEB ? (((a.order - 1) & 1) ? V_Z1 : V_Z0) : V_W0;
            const int par = S.it & 1;
            const int pold = par ? V_P0 : V_P1;
            const int pn = par ? V_P1 : V_P0;
            const float beta = (float)S.beta;
            auto pf = [&](int c) { return __fadd_rn(X(wA, c), __fmul_rn(beta, X(pold, c))); };
            double acc[1] = {0.0};
            for (int l = threadIdx.x; l < rows; l += CT)
            {
                const int row = r0 + l;
                const float pr = __fadd_rn(V(wA)[l], __fmul_rn(beta, V(pold)[l]));
                const float y = crow(a.A, row, __fmul_rn(__ldg(a.diag + row), pr), pf);
                V(pn)[l] = pr;
                V(V_Q)[l] = y;
                acc[0] += (double)pr * (double)y;
            }
            cluster_sum<1>(acc, sh, slot, cl, a.cs);
            slot ^= 1;
            if (threadIdx.x == 0)
            {
                S.wApA = acc[0];
                S.alpha = S.wArA / S.wApA;
            }
            __syncthreads();
        }
        // delta_next = delta + alpha p; rA -= alpha q; sum|rA|; next apply
        {
            const int par = S.it & 1;
            const int pv = par ? V_P1 : V_P0;
            const int dc = V_D0 + S.cur;
            const int dn = V_D0 + S.nxt;
            const float alpha = (float)S.alpha;
            double acc[2] = {0.0, 0.0};
            for (int l = threadIdx.x; l < rows; l += CT)
            {
                const int row = r0 + l;
                V(dn)[l] = __fadd_rn(V(dc)[l], __fmul_rn(alpha, V(pv)[l]));
                const float rn = __fsub_rn(V(V_RA)[l], __fmul_rn(alpha, V(V_Q)[l]));
                V(V_RA)[l] = rn;
                acc[0] += (double)fabsf(rn);
                if (CHEB)
                {
                    V(V_W0)[l] = __fmul_rn(__fmul_rn(c1, __ldg(a.rD + row)), rn);
                }
                else
                {
                    const float wa = __fmul_rn(rn, __ldg(a.rD + row));
                    V(V_W0)[l] = wa;
                    acc[1] += (double)wa * (double)rn;
                }
            }
            cluster_sum<2>(acc, sh, slot, cl, a.cs);
            slot ^= 1;
            if (threadIdx.x == 0)
            {
                S.res = acc[0];
                if (!CHEB)
                {
                    S.wArAold = S.wArA;
                    S.wArA = acc[1];
                    S.beta = S.wArA / S.wArAold;
                }
                S.cur = S.nxt;
                S.it = S.it + 1;
                inner_sync_point(&S, true);
            }
            __syncthreads();
        }
    }
    // no CTA leaves while another may still read its shared memory
    cl.sync();
    for (int l = threadIdx.x; l < rows; l += CT)
    {
        a.D[(size_t)S.cur * a.n + r0 + l] = V(V_D0 + S.cur)[l];
        if (S.best != S.cur) a.D[(size_t)S.best * a.n + r0 + l] = V(V_D0 + S.best)[l];
    }
    if (rank == 0 && threadIdx.x == 0) *a.st = S;
}

}  // namespace

namespace cf {

int cluster_shift(int n)
{
    int shift = 5;
    while (((long long)n + (1 << shift) - 1) >> shift > 16) ++shift;
    return shift;
}

int cluster_inner(cf_context* c, int order, int maxCells, bool* ran)
{
    *ran = false;
    // one row per thread (at most 16 x 1024 rows) and columns mostly in the
    // own CTA: measured on B200, several rows per thread or a mesh numbered
    // without locality (remote gathers through distributed shared memory)
    // run slower than the graph path -- e.g. 3-D 40^3 with RCM, 4 rows per
    // thread: 6.7 ms vs 2.5 ms; randomly numbered 24^3: 4.8 ms vs 1.8 ms
    if (c->n > 16 * CT || c->clusterRemote > 0.25) return CF_OK;
    const int n = c->n;
    const int shift = c->clusterShift;
    const int rpc = 1 << shift;
    const int cs = (n + rpc - 1) / rpc;
    const size_t smem = sizeof(float) * NVEC * (size_t)rpc;
    const void* fn = order > 1 ? (const void*)kc_pcg<true> : (const void*)kc_pcg<false>;
    // the attribute is the function's, shared by every context of the
    // process: always the largest value (one row per thread of a full CTA),
    // so a concurrent solve on another thread never lowers it under this
    // launch
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(sizeof(float) * NVEC * (size_t)CT)) != cudaSuccess ||
        cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)
    {
        cudaGetLastError();
        return CF_OK;
    }
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)cs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3((unsigned)cs);
    cfg.blockDim = dim3(CT);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = c->stream;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, fn, &cfg) != cudaSuccess || clusters < 1)
    {
        cudaGetLastError();
        return CF_OK;
    }
    CArgs a;
    a.A = sell_of(c);
    a.diag = c->d_diag32;
    a.rD = c->d_rD32;
    a.chebC = c->d_chebC;
    a.rA = c->d_rA;
    a.W0 = c->d_W0;
    a.st = c->d_st;
    a.D = c->d_D;
    a.n = n;
    a.order = order;
    a.shift = shift;
    a.cs = cs;
    cudaError_t e = order > 1 ? cudaLaunchKernelEx(&cfg, kc_pcg<true>, a)
                              : cudaLaunchKernelEx(&cfg, kc_pcg<false>, a);
    if (e != cudaSuccess)
        return fail(CF_ERR_CUDA, std::string("cluster launch: ") + cudaGetErrorString(e));
    c->launches++;
    *ran = true;
    return CF_OK;
}

}  // namespace cf
