// cf_coupled.cu -- one subdomain of a decomposed mesh, solved together with
// its neighbours across processor interfaces.
//
// The reference rejects coupled interfaces (metalFoamSolver.C:89-99): a
// decomposed case cannot use its GPU path.  Here a subdomain holds its own
// LDU matrix plus processor interfaces in OpenFOAM's form -- interface p
// couples cells faceCells[p][k] with the cells across face k of the
// neighbouring subdomain, and row faceCells[p][k] of A psi gets
// -coeffs[p][k] * psi_neighbour[k] (lduMatrix::Amul's
// updateMatrixInterfaces with interfaceBouCoeffs), added after the internal
// faces.
//
// Layout: the neighbours' values are a halo appended to every vector that
// an SpMV reads (x[n + haloOff[p] + k] = neighbour's value across face k of
// interface p); each interface face is one more entry of its row, after the
// row's losort faces, with column n + haloOff[p] + k and value -coeff.  So
// every row sums its internal faces in the single-domain order and then its
// interface faces in interface order, in FP32 and in FP64, as OpenFOAM's
// Amul does.
//
// Iteration: the single-domain inner loops finish every reduction inside
// the kernel that produces it; here each reduction ends in a per-subdomain
// sum, the caller's communication sums it over all subdomains (cf_comm:
// MPI/Pstream in an OpenFOAM adapter, NCCL between GPUs, or threads of one
// process), and a one-thread kernel applies the reference's scalar
// updates.  Before every SpMV the halo of its input vector is exchanged
// (gathered into a send buffer, then cf_comm.exchange).  Every kernel runs
// on the grid of its single-domain counterpart with the same per-row
// arithmetic, so a subdomain without interfaces whose communication is the
// identity returns bit for bit what cf_solve returns.  Decisions depend
// only on globally reduced values, so every subdomain takes the same steps
// (the same collectives in the same order).  One host synchronisation per
// inner iteration reads the stopping state.
#include "cudafoam.h"
#include "cf_host.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <mutex>
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

#define CF_LAUNCH()                                                             \
    do                                                                          \
    {                                                                           \
        cudaError_t e_ = cudaGetLastError();                                    \
        if (e_ != cudaSuccess)                                                  \
            return fail(CF_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e_)); \
        d->launches++;                                                          \
    } while (0)

struct cf_subdomain
{
    int device = 0;
    int numSMs = 1;
    int maxBlocksPerSM = 8;
    cudaStream_t ownStream = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::map<const void*, int> occ;
    long long launches = 0;

    bool hasTopo = false;
    bool hasCoeffs = false;
    bool hasLower = false;
    int n = 0, nf = 0, nIf = 0, nH = 0, nX = 0;   // nX = n + nH (vector length with halo)
    int nslices = 0, ellW = 0;
    long long nnzp = 0;
    int val32Sym = -1;
    std::vector<int32_t> nbr, nFaces, haloOff;
    std::vector<int32_t> perm;
    std::vector<void*> allocs;

    int* d_sliceOff = nullptr;
    int* d_col = nullptr;
    int* d_eface = nullptr;
    int* d_perm = nullptr;
    int* d_sendRow = nullptr;        // [nH] internal row of each interface face
    float* d_val32 = nullptr;
    double* d_val64 = nullptr;
    double* d_valT64 = nullptr;
    double* d_upperX = nullptr;      // [nf + nH]: upper, then -interface coefficients
    double* d_lowerX = nullptr;      // [nf + nH]: lower (or upper), then the same
    double* d_diagIn = nullptr;
    double* d_diag64 = nullptr;
    double* d_u = nullptr;
    float* d_diag32 = nullptr;
    float* d_rD32 = nullptr;
    double* d_psi = nullptr;         // [nX]
    double* d_b = nullptr;
    double* d_r64 = nullptr;
    double* d_io64 = nullptr;
    float* d_rA = nullptr;
    float* d_W0 = nullptr;           // [nX]
    float* d_W1 = nullptr;           // [nX]
    float* d_Z0 = nullptr;           // [nX]
    float* d_Z1 = nullptr;           // [nX]
    float* d_P = nullptr;            // [2 nX]
    float* d_Q = nullptr;
    float* d_T = nullptr;
    float* d_D = nullptr;            // [3 n]
    float* d_send32 = nullptr;       // [nH]
    double* d_send64 = nullptr;      // [nH]
    double* h_send = nullptr;        // [nH] pinned staging of host-buffer communication
    double* h_recv = nullptr;        // [nH]
    double* d_part = nullptr;
    InnerState* d_st = nullptr;
    DriverState* d_drv = nullptr;
    float* d_chebC = nullptr;
    double* d_sums = nullptr;        // [8] per-subdomain sums handed to the communication
    double* d_census = nullptr;      // [2] rows with non-zero row sum, sign flips
    InnerState* h_st = nullptr;
    DriverState* h_drv = nullptr;
    double* h_sums = nullptr;
};

namespace {

constexpr int MW = MAXW_UNROLL;

template <class T>
int sd_alloc(cf_subdomain* d, T** p, size_t count)
{
    *p = nullptr;
    const cudaError_t e = cudaMalloc((void**)p, std::max<size_t>(count, 1) * sizeof(T));
    if (e != cudaSuccess) return fail(CF_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    d->allocs.push_back((void*)*p);
    return CF_OK;
}

void free_topology(cf_subdomain* d)
{
    for (void* p : d->allocs) cudaFree(p);
    d->allocs.clear();
    if (d->h_send) cudaFreeHost(d->h_send);
    if (d->h_recv) cudaFreeHost(d->h_recv);
    d->h_send = d->h_recv = nullptr;
    d->hasTopo = d->hasCoeffs = false;
}

// the single-domain launch rule (grid_for): resident capacity of the kernel
// at NT threads, at most one block per NT rows
int grid_of(cf_subdomain* d, const void* fn, long long work)
{
    int occ = 0;
    auto it = d->occ.find(fn);
    if (it == d->occ.end())
    {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, NT, 0) != cudaSuccess) occ = 1;
        occ = std::max(1, std::min(occ, d->maxBlocksPerSM));
        d->occ[fn] = occ;
    }
    else
    {
        occ = it->second;
    }
    const long long cap = (long long)d->numSMs * occ;
    const long long need = (work + NT - 1) / NT;
    return (int)std::max(1LL, std::min(cap, need));
}

DevSell sell_sd(const cf_subdomain* d)
{
    DevSell A;
    A.n = d->n;
    A.nslices = d->nslices;
    A.sliceOff = d->d_sliceOff;
    A.col = d->d_col;
    A.val = d->d_val32;
    A.val64 = d->d_val64;
    A.col16 = nullptr;      // halo columns lie beyond any 16-bit row offset
    A.ellW = d->ellW;
    return A;
}

// Inner-solve buffers with P's parity blocks nX apart (the kernels of
// cf_kernels.cuh that read PcgBufs here do not touch P).
PcgBufs pcg_sd(const cf_subdomain* d)
{
    PcgBufs B;
    B.rA = d->d_rA;
    B.W0 = d->d_W0;
    B.W1 = d->d_W1;
    B.Z0 = d->d_Z0;
    B.Z1 = d->d_Z1;
    B.P = d->d_P;
    B.Q = d->d_Q;
    B.D = d->d_D;
    B.diag = d->d_diag32;
    B.rD = d->d_rD32;
    B.chebC = d->d_chebC;
    B.r64 = d->d_r64;
    B.n = d->n;
    return B;
}

// ------------------------------------------------------------------ kernels

// Per-subdomain sums: the grid_sum fold of cf_kernels.cuh, totals to `out`.
template <int NR>
__device__ __forceinline__ void sums_to(double (&acc)[NR], double* out, double* part,
                                        unsigned int* ticket)
{
    if (grid_sum<NR>(acc, part, ticket) && threadIdx.x == 0)
    {
#pragma unroll
        for (int r = 0; r < NR; ++r) out[r] = acc[r];
    }
}

template <class T>
__global__ void kc_gather_send(int nH, const int* __restrict__ row, const T* __restrict__ x,
                               T* __restrict__ send)
{
    for (int h = blockIdx.x * NT + threadIdx.x; h < nH; h += gridDim.x * NT) send[h] = x[row[h]];
}

// sum of x (k_mean_f64's partial)
__global__ void __launch_bounds__(NT) kc_sum(int n, const double* __restrict__ x, double* out,
                                             unsigned int* ticket, double* part)
{
    double acc[1] = {0.0};
    CF_ROWS(row, n) acc[0] += x[row];
    sums_to<1>(acc, out, part, ticket);
}

__global__ void __launch_bounds__(NT) kc_sum_delta(int n, const float* __restrict__ D,
                                                   const InnerState* st, double* out,
                                                   unsigned int* ticket, double* part)
{
    const float* dl = D + (size_t)st->sel * n;
    double acc[1] = {0.0};
    CF_ROWS(row, n) acc[0] += (double)dl[row];
    sums_to<1>(acc, out, part, ticket);
}

// u = A 1 including the interface coefficients, and the deflation census
// (k_sumA)
template <int MAXW>
__global__ void __launch_bounds__(NT) kc_sumA(DevSell A, const double* __restrict__ diag64,
                                              double* __restrict__ u, double* out,
                                              unsigned int* ticket, double* part)
{
    double acc[2] = {0.0, 0.0};
    CF_ROWS(row, A.n)
    {
        const double dg = diag64[row];
        const double s = row_f64<MAXW>(A, A.val64, row, dg, [](int) { return 1.0; });
        u[row] = s;
        if (fabs(s) > 1e-8 * fabs(dg)) acc[0] += 1.0;
        const double d0 = __dsub_rn(dg, s);
        if (__dmul_rn(d0, dg) <= VSMALL * fabs(d0)) acc[1] += 1.0;
    }
    sums_to<2>(acc, out, part, ticket);
}

// Gershgorin row maximum (k_gershgorin) over internal and interface entries
template <int MAXW>
__global__ void __launch_bounds__(NT) kc_gershgorin(DevSell A, const int* __restrict__ eface,
                                                    const double* __restrict__ upperX,
                                                    const double* __restrict__ diag64,
                                                    const double* __restrict__ u, int deflate,
                                                    double* out, unsigned int* ticket,
                                                    double* part)
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
            if (is_nbr(c)) so = __dadd_rn(so, fabs(upperX[eface[base + SLICE * k]]));
        }
        for (int k = 0; k < w; ++k)
        {
            const int c = A.col[base + SLICE * k];
            if (is_own(c)) so = __dadd_rn(so, fabs(upperX[eface[base + SLICE * k]]));
        }
        const double dp = deflate ? __dsub_rn(diag64[row], u[row]) : diag64[row];
        m = fmax(m, __dadd_rn(1.0, so / fabs(dp)));
    }
    if (grid_max(m, part, ticket) && threadIdx.x == 0) *out = m;
}

// r = b - A psi, normFactor partial and sum|r| (k_residual0); psi carries its halo
template <int MAXW>
__global__ void __launch_bounds__(NT) kc_residual0(DevSell A, const double* __restrict__ diag64,
                                                   const double* __restrict__ psi,
                                                   const double* __restrict__ b,
                                                   const double* __restrict__ u,
                                                   double* __restrict__ r64,
                                                   const DriverState* drv, double* out,
                                                   unsigned int* ticket, double* part)
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
    sums_to<2>(acc, out, part, ticket);
}

// r = b - A psi; u.r and u.u (deflating) or sum|r| (k_residual)
template <int MAXW>
__global__ void __launch_bounds__(NT) kc_residual(DevSell A, const double* __restrict__ diag64,
                                                  const double* __restrict__ psi,
                                                  const double* __restrict__ b,
                                                  const double* __restrict__ u,
                                                  double* __restrict__ r64, int deflate,
                                                  double* out, unsigned int* ticket, double* part)
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
    sums_to<2>(acc, out, part, ticket);
}

// psi += c, r -= c u, then sum|r| (k_cshift, c from the global u.r, u.u)
__global__ void __launch_bounds__(NT) kc_cshift(int n, double* __restrict__ psi,
                                                double* __restrict__ r64,
                                                const double* __restrict__ u,
                                                const DriverState* drv, double* out,
                                                unsigned int* ticket, double* part)
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
    sums_to<1>(acc, out, part, ticket);
}

__global__ void __launch_bounds__(NT) kc_l2(int n, const double* __restrict__ r64,
                                            const double* __restrict__ b, double* out,
                                            unsigned int* ticket, double* part)
{
    double acc[2] = {0.0, 0.0};
    CF_ROWS(row, n)
    {
        acc[0] += r64[row] * r64[row];
        acc[1] += b[row] * b[row];
    }
    sums_to<2>(acc, out, part, ticket);
}

// driver finalisers: one thread, the single-domain finalisers' arithmetic on
// the global sums
enum
{
    FIN_XBAR, FIN_RES0, FIN_RES, FIN_CSHIFT, FIN_L2, FIN_RMEAN, FIN_DMEAN, FIN_CENSUS, FIN_CHEB
};

__global__ void kc_fin_driver(int what, const double* g, double nGlobal, DriverState* drv,
                              int deflate, int order, double ratio, float* chebC)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    switch (what)
    {
        case FIN_XBAR: drv->xbar = g[0] / nGlobal; break;
        case FIN_RES0:
            drv->normFactor = g[0] + 1e-20;
            drv->initRes = g[1] / drv->normFactor;
            drv->finalRes = drv->initRes;
            break;
        case FIN_RES:
            if (deflate)
            {
                drv->ur = g[0];
                drv->uu = g[1];
            }
            else
            {
                drv->finalRes = g[0] / drv->normFactor;
            }
            break;
        case FIN_CSHIFT: drv->finalRes = g[0] / drv->normFactor; break;
        case FIN_L2:
            drv->l2r = sqrt(g[0]);
            drv->l2b = sqrt(g[1]);
            break;
        case FIN_RMEAN: drv->rmean = g[0] / nGlobal; break;
        case FIN_DMEAN: drv->dmean = g[0] / nGlobal; break;
        case FIN_CENSUS:
            drv->nPinned = (long long)g[0];
            drv->signflip = g[1] > 0.0;
            break;
        case FIN_CHEB:
            drv->chebBeta = g[0];
            cheb_constants(order, g[0], ratio, chebC);
            break;
    }
}

// -------------------------------------------------------------- inner PCG

// k_pcg_init with P's parity blocks nX apart; Jacobi: wA.rA partial
template <bool CHEB>
__global__ void __launch_bounds__(NT) kc_pcg_init(PcgBufs B, int nX, const double* mean,
                                                  double* out, unsigned int* ticket, double* part)
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
        B.P[nX + row] = 0.0f;
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
    if (!CHEB) sums_to<1>(acc, out, part, ticket);
}

// the last Chebyshev step (k_cheb_step<true>) with its z.r partial
template <int MAXW>
__global__ void __launch_bounds__(NT) kc_cheb_last(DevSell A, PcgBufs B, const float* zin,
                                                   const float* win, float* wout, float* zout,
                                                   int j, const InnerState* st, double* out,
                                                   unsigned int* ticket, double* part)
{
    if (st->done) return;
    const float c2 = B.chebC[2 * j - 1];
    const float c3 = B.chebC[2 * j];
    double acc[1] = {0.0};
    CF_ROWS(row, A.n)
    {
        const float zr = zin[row];
        const float v = row_f32<MAXW>(A, row, __fmul_rn(B.diag[row], zr),
                                      [&](int c) { return __ldg(zin + c); });
        const float r = B.rA[row];
        const float wn = __fadd_rn(__fmul_rn(c2, win[row]),
                                   __fmul_rn(__fmul_rn(c3, B.rD[row]), __fsub_rn(r, v)));
        const float zn = __fadd_rn(zr, wn);
        wout[row] = wn;
        zout[row] = zn;
        acc[0] += (double)zn * (double)r;
    }
    sums_to<1>(acc, out, part, ticket);
}

// p = wA + beta p_old (the p-update k_pcg_p_spmv forms at its gathers)
__global__ void kc_p_update(int n, const float* __restrict__ wA, const float* __restrict__ Pold,
                            float* __restrict__ Pn, const InnerState* st)
{
    if (st->done) return;
    const float beta = (float)st->beta;
    CF_ROWS(row, n) Pn[row] = __fadd_rn(wA[row], __fmul_rn(beta, Pold[row]));
}

// y = A x over the halo-extended x, and w.y partial
template <int MAXW>
__global__ void __launch_bounds__(NT) kc_spmv_dot(DevSell A, const float* __restrict__ diag,
                                                  const float* __restrict__ x,
                                                  float* __restrict__ y,
                                                  const float* __restrict__ w,
                                                  const InnerState* st, double* out,
                                                  unsigned int* ticket, double* part)
{
    if (st->done) return;
    double acc[1] = {0.0};
    CF_ROWS(row, A.n)
    {
        const float v = row_f32<MAXW>(A, row, __fmul_rn(diag[row], x[row]),
                                      [&](int c) { return __ldg(x + c); });
        y[row] = v;
        acc[0] += (double)w[row] * (double)v;
    }
    sums_to<1>(acc, out, part, ticket);
}

// k_pcg_update's vector work with P's parity blocks nX apart
template <bool CHEB>
__global__ void __launch_bounds__(NT) kc_pcg_update(PcgBufs B, int nX, const InnerState* st,
                                                    double* out, unsigned int* ticket,
                                                    double* part)
{
    if (st->done) return;
    const int n = B.n;
    const float* __restrict__ P = B.P + (size_t)(st->it & 1) * nX;
    const float* __restrict__ D = B.D + (size_t)st->cur * n;
    float* __restrict__ Dn = B.D + (size_t)st->nxt * n;
    const float alpha = (float)st->alpha;
    const float c1 = CHEB ? B.chebC[0] : 0.0f;
    double acc[2] = {0.0, 0.0};
    CF_ROWS(row, n)
    {
        Dn[row] = __fadd_rn(D[row], __fmul_rn(alpha, P[row]));
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
    sums_to<2>(acc, out, part, ticket);
}

// ---------------------------------------------------------- inner BiCGStab

__global__ void __launch_bounds__(NT) kc_bicg_init(BicgBufs B, double* out, unsigned int* ticket,
                                                   double* part)
{
    double acc[1] = {0.0};
    CF_ROWS(row, B.n)
    {
        const float ra = (float)B.r64[row];
        B.rA[row] = ra;
        B.rA0[row] = ra;
        B.D[row] = 0.0f;
        B.P[row] = 0.0f;
        B.AyA[row] = 0.0f;
        acc[0] += (double)ra * (double)ra;
    }
    sums_to<1>(acc, out, part, ticket);
}

// p = rA + beta (p - omega AyA), yA = rD p (bicg_update_p + emul)
__global__ void kc_bicg_p(BicgBufs B, const InnerState* st)
{
    if (st->done) return;
    const float beta = (float)st->beta;
    const float omega = (float)st->omega;
    CF_ROWS(row, B.n)
    {
        const float p = __fadd_rn(B.rA[row],
                                  __fmul_rn(beta, __fsub_rn(B.P[row], __fmul_rn(omega, B.AyA[row]))));
        B.P[row] = p;
        B.yA[row] = __fmul_rn(B.rD[row], p);
    }
}

// s = rA - alpha AyA, zA = rD s, sum|s| partial (bicg_s_res + emul)
__global__ void __launch_bounds__(NT) kc_bicg_s(BicgBufs B, const InnerState* st, double* out,
                                                unsigned int* ticket, double* part)
{
    if (st->done) return;
    const float alpha = (float)st->alpha;
    double acc[1] = {0.0};
    CF_ROWS(row, B.n)
    {
        const float sv = __fsub_rn(B.rA[row], __fmul_rn(alpha, B.AyA[row]));
        B.sA[row] = sv;
        B.zA[row] = __fmul_rn(B.rD[row], sv);
        acc[0] += (double)fabsf(sv);
    }
    sums_to<1>(acc, out, part, ticket);
}

// tA = A zA over the halo-extended zA; s.tA and tA.tA partials
template <int MAXW>
__global__ void __launch_bounds__(NT) kc_bicg_t(DevSell A, BicgBufs B, const InnerState* st,
                                                double* out, unsigned int* ticket, double* part)
{
    if (st->done) return;
    double acc[2] = {0.0, 0.0};
    CF_ROWS(row, A.n)
    {
        const float t = row_f32<MAXW>(A, row, __fmul_rn(B.diag[row], B.zA[row]),
                                      [&](int c) { return __ldg(B.zA + c); });
        B.tA[row] = t;
        const float sv = B.sA[row];
        acc[0] += (double)sv * (double)t;
        acc[1] += (double)t * (double)t;
    }
    sums_to<2>(acc, out, part, ticket);
}

// bicg_update_sol_res, or the early-exit update, with sum|rA| and rA0.rA
__global__ void __launch_bounds__(NT) kc_bicg_e(BicgBufs B, const InnerState* st, double* out,
                                                unsigned int* ticket, double* part)
{
    const bool early = st->early;
    if ((st->done && !early) || st->converged) return;
    const int n = B.n;
    const float alpha = (float)st->alpha;
    const float* __restrict__ D = B.D + (size_t)st->cur * n;
    float* __restrict__ Dn = B.D + (size_t)st->nxt * n;
    double acc[2] = {0.0, 0.0};
    if (early)
    {
        CF_ROWS(row, n) Dn[row] = __fadd_rn(D[row], __fmul_rn(alpha, B.yA[row]));
    }
    else
    {
        const float omega = (float)st->omega;
        CF_ROWS(row, n)
        {
            Dn[row] = __fadd_rn(D[row], __fadd_rn(__fmul_rn(alpha, B.yA[row]),
                                                  __fmul_rn(omega, B.zA[row])));
            const float r = __fsub_rn(B.sA[row], __fmul_rn(omega, B.tA[row]));
            B.rA[row] = r;
            acc[0] += (double)fabsf(r);
            acc[1] += (double)B.rA0[row] * (double)r;
        }
    }
    sums_to<2>(acc, out, part, ticket);
}

// inner finalisers: the single-domain kernels' last-block updates on the
// global sums
enum
{
    IN_PCG_INIT, IN_CHEB_LAST, IN_ALPHA_PCG, IN_PCG_UPDATE_CHEB, IN_PCG_UPDATE_JACOBI,
    IN_BICG_INIT, IN_ALPHA_BICG, IN_OMEGA, IN_BICG_E
};

__global__ void kc_fin_inner(int what, const double* g, InnerState* st)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    switch (what)
    {
        case IN_PCG_INIT:
            st->wArAold = st->wArA;
            st->wArA = g[0];
            st->beta = 0.0;
            break;
        case IN_CHEB_LAST:
            if (st->done) return;
            st->wArAold = st->wArA;
            st->wArA = g[0];
            st->beta = (st->it == 0) ? 0.0 : st->wArA / st->wArAold;
            break;
        case IN_ALPHA_PCG:
            if (st->done) return;
            st->wApA = g[0];
            st->alpha = st->wArA / st->wApA;
            break;
        case IN_PCG_UPDATE_CHEB:
        case IN_PCG_UPDATE_JACOBI:
            if (st->done) return;
            st->res = g[0];
            if (what == IN_PCG_UPDATE_JACOBI)
            {
                st->wArAold = st->wArA;
                st->wArA = g[1];
                st->beta = st->wArA / st->wArAold;
            }
            st->cur = st->nxt;
            st->it = st->it + 1;
            inner_sync_point(st, true);
            break;
        case IN_BICG_INIT:
            st->rA0rAold = st->rA0rA;
            st->rA0rA = g[0];
            st->beta = 0.0;
            break;
        case IN_ALPHA_BICG:
            if (st->done) return;
            st->rA0AyA = g[0];
            st->alpha = st->rA0rA / st->rA0AyA;
            break;
        case IN_OMEGA:   // g = sum|s|, s.t, t.t
            if (st->done) return;
            st->resS = g[0];
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
                st->tAsA = g[1];
                st->tAtA = g[2];
                st->omega = st->tAsA / st->tAtA;
            }
            break;
        case IN_BICG_E:
            if ((st->done && !st->early) || st->converged) return;
            if (st->early)
            {
                st->cur = st->nxt;
                st->it = st->it + 1;
                st->finalResSum = st->resS;
                st->converged = 1;
                return;
            }
            st->res = g[0];
            st->cur = st->nxt;
            st->it = st->it + 1;
            inner_sync_point(st, false);
            st->rA0rAold = st->rA0rA;
            st->rA0rA = g[1];
            st->beta = (st->rA0rA / st->rA0rAold) * (st->alpha / st->omega);
            break;
    }
}

// ------------------------------------------------------------------ host

struct Ctx
{
    cf_subdomain* d;
    const cf_comm* comm;
};

// global sums of `count` per-subdomain values at d_sums (in place)
int allreduce(Ctx& x, int count, int op)
{
    cf_subdomain* d = x.d;
    double* buf = d->d_sums;
    if (x.comm->hostBuffers)
    {
        CF_CUDA(cudaMemcpyAsync(d->h_sums, d->d_sums, sizeof(double) * count,
                                cudaMemcpyDeviceToHost, d->stream));
        CF_CUDA(cudaStreamSynchronize(d->stream));
        buf = d->h_sums;
    }
    const int rc = x.comm->allreduce(x.comm->user, buf, count, op, (void*)d->stream);
    if (rc != 0) return fail(CF_ERR_CUDA, "cf_comm.allreduce failed (" + std::to_string(rc) + ")");
    if (x.comm->hostBuffers)
        CF_CUDA(cudaMemcpyAsync(d->d_sums, d->h_sums, sizeof(double) * count,
                                cudaMemcpyHostToDevice, d->stream));
    return CF_OK;
}

// neighbours' values into the halo of x (FP32 or FP64)
template <class T>
int exchange(Ctx& x, T* vec)
{
    cf_subdomain* d = x.d;
    if (d->nIf == 0) return CF_OK;
    T* send = std::is_same<T, float>::value ? (T*)d->d_send32 : (T*)d->d_send64;
    kc_gather_send<T><<<std::max(1, std::min((d->nH + NT - 1) / NT, d->numSMs * 4)), NT, 0,
                        d->stream>>>(d->nH, d->d_sendRow, vec, send);
    CF_LAUNCH();
    const bool host = x.comm->hostBuffers != 0;
    T* hs = reinterpret_cast<T*>(d->h_send);
    T* hr = reinterpret_cast<T*>(d->h_recv);
    if (host)
    {
        CF_CUDA(cudaMemcpyAsync(hs, send, sizeof(T) * d->nH, cudaMemcpyDeviceToHost, d->stream));
        CF_CUDA(cudaStreamSynchronize(d->stream));
    }
    std::vector<const void*> s(d->nIf);
    std::vector<void*> r(d->nIf);
    for (int p = 0; p < d->nIf; ++p)
    {
        s[p] = host ? (const void*)(hs + d->haloOff[p]) : (const void*)(send + d->haloOff[p]);
        r[p] = host ? (void*)(hr + d->haloOff[p]) : (void*)(vec + d->n + d->haloOff[p]);
    }
    const int rc = x.comm->exchange(x.comm->user, d->nIf, d->nbr.data(), d->nFaces.data(),
                                    (int32_t)sizeof(T), s.data(), r.data(), (void*)d->stream);
    if (rc != 0) return fail(CF_ERR_CUDA, "cf_comm.exchange failed (" + std::to_string(rc) + ")");
    if (host)
        CF_CUDA(cudaMemcpyAsync(vec + d->n, hr, sizeof(T) * d->nH, cudaMemcpyHostToDevice,
                                d->stream));
    return CF_OK;
}

int fin_driver(Ctx& x, int what, double nGlobal, int deflate = 0, int order = 1,
               double ratio = 30.0)
{
    cf_subdomain* d = x.d;
    kc_fin_driver<<<1, 32, 0, d->stream>>>(what, d->d_sums, nGlobal, d->d_drv, deflate, order,
                                           ratio, d->d_chebC);
    CF_LAUNCH();
    return CF_OK;
}

int fin_inner(Ctx& x, int what)
{
    cf_subdomain* d = x.d;
    kc_fin_inner<<<1, 32, 0, d->stream>>>(what, d->d_sums, d->d_st);
    CF_LAUNCH();
    return CF_OK;
}

int fetch_drv(cf_subdomain* d)
{
    CF_CUDA(cudaMemcpyAsync(d->h_drv, d->d_drv, sizeof(DriverState), cudaMemcpyDeviceToHost,
                            d->stream));
    CF_CUDA(cudaStreamSynchronize(d->stream));
    return CF_OK;
}

int fetch_st(cf_subdomain* d)
{
    CF_CUDA(cudaMemcpyAsync(d->h_st, d->d_st, sizeof(InnerState), cudaMemcpyDeviceToHost,
                            d->stream));
    CF_CUDA(cudaStreamSynchronize(d->stream));
    return CF_OK;
}

int stage_vals_sd(cf_subdomain* d, int sym32)
{
    const double* lo = d->hasLower ? d->d_lowerX : d->d_upperX;
    const int g = grid_of(d, (const void*)k_stage_vals, d->nnzp);
    k_stage_vals<<<g, NT, 0, d->stream>>>(d->nnzp, d->d_col, d->d_eface, d->d_upperX, lo, sym32,
                                          d->d_val32, d->d_val64, d->d_valT64);
    CF_LAUNCH();
    d->val32Sym = sym32;
    return CF_OK;
}

int stage_diag32_sd(cf_subdomain* d, int deflate)
{
    k_stage_diag32<<<grid_of(d, (const void*)k_stage_diag32, d->n), NT, 0, d->stream>>>(
        d->n, d->d_diag64, d->d_u, deflate, d->d_diag32, d->d_rD32);
    CF_LAUNCH();
    return CF_OK;
}

// One inner FP32 PCG (Chebyshev-Jacobi of `order`, Jacobi for 1) or
// BiCGStab (Jacobi) on the subdomain's part of A delta = r.
int inner_solve(Ctx& x, bool bicg, const double* mean, double target, int maxIter, int ips,
                int order, int stagLimit, cf_inner_stats* out)
{
    cf_subdomain* d = x.d;
    cudaStream_t s = d->stream;
    const int n = d->n;
    const DevSell A = sell_sd(d);
    const PcgBufs B = pcg_sd(d);
    BicgBufs Bb;
    Bb.rA = d->d_rA;
    Bb.rA0 = d->d_W0;
    Bb.P = d->d_P;
    Bb.yA = d->d_W1;
    Bb.AyA = d->d_Q;
    Bb.sA = d->d_Z0;
    Bb.zA = d->d_Z1;
    Bb.tA = d->d_T;
    Bb.D = d->d_D;
    Bb.diag = d->d_diag32;
    Bb.rD = d->d_rD32;
    Bb.r64 = d->d_r64;
    Bb.n = n;
    unsigned int* tk = &d->d_st->ticket;
    double* g = d->d_sums;
    k_inner_setup<<<1, 32, 0, s>>>(d->d_st, target, maxIter, ips, stagLimit);
    CF_LAUNCH();
    if (!bicg)
    {
        if (order > 1)
        {
            kc_pcg_init<true><<<grid_of(d, (const void*)k_pcg_init<true>, n), NT, 0, s>>>(
                B, d->nX, mean, g, tk, d->d_part);
            CF_LAUNCH();
        }
        else
        {
            kc_pcg_init<false><<<grid_of(d, (const void*)k_pcg_init<false>, n), NT, 0, s>>>(
                B, d->nX, mean, g, tk, d->d_part);
            CF_LAUNCH();
            CF_TRY(allreduce(x, 1, 0));
            CF_TRY(fin_inner(x, IN_PCG_INIT));
        }
    }
    else
    {
        kc_bicg_init<<<grid_of(d, (const void*)k_bicg_init, n), NT, 0, s>>>(Bb, g, tk, d->d_part);
        CF_LAUNCH();
        CF_TRY(allreduce(x, 1, 0));
        CF_TRY(fin_inner(x, IN_BICG_INIT));
    }
    CF_CUDA(cudaEventRecord(d->ev0, s));
    for (int it = 0; it < maxIter; ++it)
    {
        if (!bicg)
        {
            const float* wA = B.W0;
            if (order > 1)
            {
                float* Z[2] = {B.Z0, B.Z1};
                for (int j = 1; j < order; ++j)
                {
                    float* zin = (j == 1) ? B.W0 : Z[(j - 1) & 1];
                    const float* win = (j == 1) ? B.W0 : B.W1;
                    CF_TRY(exchange<float>(x, zin));
                    if (j == order - 1)
                    {
                        kc_cheb_last<MW><<<grid_of(d, (const void*)k_cheb_step<true, MW>, n), NT, 0,
                                           s>>>(A, B, zin, win, B.W1, Z[j & 1], j, d->d_st, g, tk,
                                                d->d_part);
                        CF_LAUNCH();
                        CF_TRY(allreduce(x, 1, 0));
                        CF_TRY(fin_inner(x, IN_CHEB_LAST));
                    }
                    else
                    {
                        auto fn = k_cheb_step<false, MW>;
                        fn<<<rows_grid(n), NT, 0, s>>>(A, B, zin, win, B.W1, Z[j & 1], j,
                                                       d->d_st, d->d_part);
                        CF_LAUNCH();
                    }
                }
                wA = Z[(order - 1) & 1];
            }
            // p (parity of the iteration), its halo, q = A p and p.q
            const int par = it & 1;
            float* Pn = d->d_P + (size_t)par * d->nX;
            const float* Pold = d->d_P + (size_t)(par ^ 1) * d->nX;
            const int gp = grid_of(d, (const void*)k_pcg_p_spmv<MW>, n);
            kc_p_update<<<gp, NT, 0, s>>>(n, wA, Pold, Pn, d->d_st);
            CF_LAUNCH();
            CF_TRY(exchange<float>(x, Pn));
            kc_spmv_dot<MW><<<gp, NT, 0, s>>>(A, B.diag, Pn, B.Q, Pn, d->d_st, g, tk, d->d_part);
            CF_LAUNCH();
            CF_TRY(allreduce(x, 1, 0));
            CF_TRY(fin_inner(x, IN_ALPHA_PCG));
            if (order > 1)
                kc_pcg_update<true><<<grid_of(d, (const void*)k_pcg_update<true>, n), NT, 0, s>>>(
                    B, d->nX, d->d_st, g, tk, d->d_part);
            else
                kc_pcg_update<false><<<grid_of(d, (const void*)k_pcg_update<false>, n), NT, 0,
                                       s>>>(B, d->nX, d->d_st, g, tk, d->d_part);
            CF_LAUNCH();
            CF_TRY(allreduce(x, 2, 0));
            CF_TRY(fin_inner(x, order > 1 ? IN_PCG_UPDATE_CHEB : IN_PCG_UPDATE_JACOBI));
        }
        else
        {
            const int gab = grid_of(d, (const void*)k_bicg_ab<MW>, n);
            const int gcd = grid_of(d, (const void*)k_bicg_cd<MW>, n);
            kc_bicg_p<<<gab, NT, 0, s>>>(Bb, d->d_st);
            CF_LAUNCH();
            CF_TRY(exchange<float>(x, Bb.yA));
            kc_spmv_dot<MW><<<gab, NT, 0, s>>>(A, Bb.diag, Bb.yA, Bb.AyA, Bb.rA0, d->d_st, g, tk,
                                               d->d_part);
            CF_LAUNCH();
            CF_TRY(allreduce(x, 1, 0));
            CF_TRY(fin_inner(x, IN_ALPHA_BICG));
            kc_bicg_s<<<gcd, NT, 0, s>>>(Bb, d->d_st, g, tk, d->d_part);
            CF_LAUNCH();
            CF_TRY(exchange<float>(x, Bb.zA));
            kc_bicg_t<MW><<<gcd, NT, 0, s>>>(A, Bb, d->d_st, g + 1, tk, d->d_part);
            CF_LAUNCH();
            CF_TRY(allreduce(x, 3, 0));
            CF_TRY(fin_inner(x, IN_OMEGA));
            kc_bicg_e<<<grid_of(d, (const void*)k_bicg_e, n), NT, 0, s>>>(Bb, d->d_st, g, tk,
                                                                          d->d_part);
            CF_LAUNCH();
            CF_TRY(allreduce(x, 2, 0));
            CF_TRY(fin_inner(x, IN_BICG_E));
        }
        CF_TRY(fetch_st(d));
        if (d->h_st->done) break;
    }
    CF_CUDA(cudaEventRecord(d->ev1, s));
    k_inner_final<<<1, 32, 0, s>>>(d->d_st);
    CF_LAUNCH();
    CF_TRY(fetch_st(d));
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, d->ev0, d->ev1);
    const InnerState& st = *d->h_st;
    out->nIterations = st.it;
    out->converged = st.converged;
    out->singular = st.singular;
    out->stagnated = st.stagnated;
    out->finalResSum = st.finalResSum;
    out->tGpuSeconds = ms * 1e-3;
    out->tWallSeconds = 0.0;
    return CF_OK;
}

bool converged_host(double tol, double relTol, double initial, double fin)
{
    return (fin < tol) || (relTol > 1e-20 && fin < relTol * initial);
}

// metalFoamSolver::solveImpl over all subdomains (the steps of
// cf_solve's driver with every sum global and psi's halo exchanged before
// each FP64 residual); psi/src host arrays in the caller's cell order.
int solve_sd(Ctx& x, int solver, double* psi, const double* src, cudaMemcpyKind kind,
             const cf_options* o, cf_performance* perf)
{
    cf_subdomain* d = x.d;
    const bool bicg = solver == CF_SOLVER_PBICGSTAB;
    cudaStream_t s = d->stream;
    const int n = d->n;
    const DevSell A = sell_sd(d);
    double* g = d->d_sums;
    unsigned int* tk = &d->d_drv->ticket;
    std::memset(perf, 0, sizeof(*perf));
    const double tw0 = wall_now();

    const int wantSym32 = (!bicg || !d->hasLower) ? 1 : 0;
    if (wantSym32 != d->val32Sym) CF_TRY(stage_vals_sd(d, wantSym32));
    CF_CUDA(cudaMemcpyAsync(d->d_io64, psi, sizeof(double) * n, kind, s));
    const int gRow = grid_of(d, (const void*)k_gather_f64, n);
    k_gather_f64<<<gRow, NT, 0, s>>>(n, d->d_perm, d->d_io64, d->d_psi);
    CF_LAUNCH();
    CF_CUDA(cudaMemcpyAsync(d->d_io64, src, sizeof(double) * n, kind, s));
    k_gather_f64<<<gRow, NT, 0, s>>>(n, d->d_perm, d->d_io64, d->d_b);
    CF_LAUNCH();

    // global cell count
    CF_TRY([&]() -> int {
        const double nl = (double)n;
        CF_CUDA(cudaMemcpyAsync(g, &nl, sizeof(double), cudaMemcpyHostToDevice, s));
        CF_CUDA(cudaStreamSynchronize(s));
        return CF_OK;
    }());
    CF_TRY(allreduce(x, 1, 0));
    CF_CUDA(cudaMemcpyAsync(d->h_sums, g, sizeof(double), cudaMemcpyDeviceToHost, s));
    CF_CUDA(cudaStreamSynchronize(s));
    const double nGlobal = d->h_sums[0];

    // initial residual and normFactor (metalFoamSolver.C:109-129)
    kc_sum<<<grid_of(d, (const void*)k_mean_f64, n), NT, 0, s>>>(n, d->d_psi, g, tk, d->d_part);
    CF_LAUNCH();
    CF_TRY(allreduce(x, 1, 0));
    CF_TRY(fin_driver(x, FIN_XBAR, nGlobal));
    CF_TRY(exchange<double>(x, d->d_psi));
    kc_residual0<MW><<<grid_of(d, (const void*)k_residual0<MW>, n), NT, 0, s>>>(
        A, d->d_diag64, d->d_psi, d->d_b, d->d_u, d->d_r64, d->d_drv, g, tk, d->d_part);
    CF_LAUNCH();
    CF_TRY(allreduce(x, 2, 0));
    CF_TRY(fin_driver(x, FIN_RES0, nGlobal));
    CF_TRY(fetch_drv(d));
    perf->normFactor = d->h_drv->normFactor;
    perf->initialResidual = d->h_drv->initRes;
    perf->finalResidual = perf->initialResidual;
    perf->chebBeta = 2.0;

    if (o->minIter > 0 ||
        !converged_host(o->tolerance, o->relTol, perf->initialResidual, perf->finalResidual))
    {
        perf->solved = 1;
        // deflation decision (metalFoamSolver.C:170-209) on the global census
        CF_CUDA(cudaMemcpyAsync(g, d->d_census, 2 * sizeof(double), cudaMemcpyDeviceToDevice, s));
        CF_TRY(allreduce(x, 2, 0));
        CF_TRY(fin_driver(x, FIN_CENSUS, nGlobal));
        CF_TRY(fetch_drv(d));
        bool deflate = false;
        if (!bicg && o->deflate != CF_DEFLATE_OFF)
            deflate = o->deflate == CF_DEFLATE_ON || 10.0 * (double)d->h_drv->nPinned <= nGlobal;
        if (deflate && d->h_drv->signflip) deflate = false;
        perf->deflated = deflate;
        CF_TRY(stage_diag32_sd(d, deflate ? 1 : 0));
        const int order = bicg ? 1 : o->chebyshevOrder;
        if (order < 1 || order > CF_MAX_CHEB)
            return fail(CF_ERR_INVALID_ARG, "chebyshevOrder must be in [1, 64]");
        if (order > 1)
        {
            kc_gershgorin<MW><<<grid_of(d, (const void*)k_gershgorin<MW>, n), NT, 0, s>>>(
                A, d->d_eface, d->d_upperX, d->d_diag64, d->d_u, deflate ? 1 : 0, g, tk,
                d->d_part);
            CF_LAUNCH();
            CF_TRY(allreduce(x, 1, 1));
            CF_TRY(fin_driver(x, FIN_CHEB, nGlobal, 0, order, o->chebyshevRatio));
            CF_TRY(fetch_drv(d));
            perf->chebBeta = d->h_drv->chebBeta;
        }
        const double target =
            std::max(o->tolerance, o->relTol * perf->initialResidual) * perf->normFactor;
        int totalIter = 0, outer = 0, singular = 0;
        double prevRes = perf->initialResidual;
        for (outer = 0; outer <= o->maxRestarts; ++outer)
        {
            const double* meanp = nullptr;
            if (deflate)
            {
                kc_sum<<<grid_of(d, (const void*)k_mean_f64, n), NT, 0, s>>>(n, d->d_r64, g, tk,
                                                                             d->d_part);
                CF_LAUNCH();
                CF_TRY(allreduce(x, 1, 0));
                CF_TRY(fin_driver(x, FIN_RMEAN, nGlobal));
                meanp = &d->d_drv->rmean;
            }
            cf_inner_stats st;
            CF_TRY(inner_solve(x, bicg, meanp, target, o->maxIter - totalIter,
                               o->iterationsPerSync, order,
                               o->stagnationLimit > 0 ? o->stagnationLimit : STAG_LIMIT, &st));
            totalIter += st.nIterations;
            perf->tGpu += st.tGpuSeconds;
            singular = st.singular;
            perf->stagnated = st.stagnated;
            perf->finalResSum32 = st.finalResSum;
            const double* dmeanp = nullptr;
            if (deflate)
            {
                kc_sum_delta<<<grid_of(d, (const void*)k_mean_delta, n), NT, 0, s>>>(
                    n, d->d_D, d->d_st, g, tk, d->d_part);
                CF_LAUNCH();
                CF_TRY(allreduce(x, 1, 0));
                CF_TRY(fin_driver(x, FIN_DMEAN, nGlobal));
                dmeanp = &d->d_drv->dmean;
            }
            k_psi_update<<<grid_of(d, (const void*)k_psi_update, n), NT, 0, s>>>(
                n, d->d_psi, d->d_D, d->d_st, dmeanp);
            CF_LAUNCH();
            CF_TRY(exchange<double>(x, d->d_psi));
            kc_residual<MW><<<grid_of(d, (const void*)k_residual<MW>, n), NT, 0, s>>>(
                A, d->d_diag64, d->d_psi, d->d_b, d->d_u, d->d_r64, deflate ? 1 : 0, g, tk,
                d->d_part);
            CF_LAUNCH();
            CF_TRY(allreduce(x, 2, 0));
            CF_TRY(fin_driver(x, FIN_RES, nGlobal, deflate ? 1 : 0));
            if (deflate)
            {
                kc_cshift<<<grid_of(d, (const void*)k_cshift, n), NT, 0, s>>>(
                    n, d->d_psi, d->d_r64, d->d_u, d->d_drv, g, tk, d->d_part);
                CF_LAUNCH();
                CF_TRY(allreduce(x, 1, 0));
                CF_TRY(fin_driver(x, FIN_CSHIFT, nGlobal));
            }
            CF_TRY(fetch_drv(d));
            perf->finalResidual = d->h_drv->finalRes;
            perf->nIterations = totalIter;
            // hybrid polish (metalFoamSolver.C:371-390)
            if (deflate && perf->finalResidual > prevRes / 1.5 && !st.singular)
            {
                deflate = false;
                perf->polished = 1;
                CF_TRY(stage_diag32_sd(d, 0));
            }
            prevRes = perf->finalResidual;
            if (o->verbose)
                std::printf("    coupled restart %d: inner=%d fp32ResSum=%g fp64Res=%g\n", outer,
                            st.nIterations, st.finalResSum, perf->finalResidual);
            if (singular) break;
            if (totalIter >= o->maxIter) break;
            if (perf->nIterations >= o->minIter &&
                converged_host(o->tolerance, o->relTol, perf->initialResidual,
                               perf->finalResidual))
                break;
        }
        perf->nRestarts = outer;
        perf->singular = singular;
    }
    perf->converged =
        converged_host(o->tolerance, o->relTol, perf->initialResidual, perf->finalResidual);
    kc_l2<<<grid_of(d, (const void*)k_l2, n), NT, 0, s>>>(n, d->d_r64, d->d_b, g, tk, d->d_part);
    CF_LAUNCH();
    CF_TRY(allreduce(x, 2, 0));
    CF_TRY(fin_driver(x, FIN_L2, nGlobal));
    k_scatter_f64<<<gRow, NT, 0, s>>>(n, d->d_perm, d->d_psi, d->d_io64);
    CF_LAUNCH();
    const cudaMemcpyKind back = kind == cudaMemcpyHostToDevice ? cudaMemcpyDeviceToHost
                                                                : cudaMemcpyDeviceToDevice;
    CF_CUDA(cudaMemcpyAsync(psi, d->d_io64, sizeof(double) * n, back, s));
    CF_TRY(fetch_drv(d));
    perf->residualL2 = d->h_drv->l2b > 0 ? d->h_drv->l2r / d->h_drv->l2b : d->h_drv->l2r;
    perf->tSolve = wall_now() - tw0;
    return CF_OK;
}

}  // namespace

// ------------------------------------------------------------------ C ABI

extern "C" int cf_subdomain_create(cf_subdomain** out, int32_t device)
{
    if (!out) return fail(CF_ERR_INVALID_ARG, "out is NULL");
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
    {
        cudaGetLastError();
        return fail(CF_ERR_NO_DEVICE, "cudaFoam: no CUDA device available");
    }
    if (device < 0 || device >= count) return fail(CF_ERR_INVALID_ARG, "device index out of range");
    cudaDeviceProp prop;
    CF_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10)
        return fail(CF_ERR_NO_DEVICE, std::string("cudaFoam: ") + prop.name +
                                          " is not an sm_100 (B200-class) device");
    CF_CUDA(cudaSetDevice(device));
    cf_subdomain* d = new cf_subdomain();
    d->device = device;
    d->numSMs = prop.multiProcessorCount;
    d->maxBlocksPerSM = std::max(1, prop.maxThreadsPerMultiProcessor / NT);
    const size_t partCount = (size_t)NPART * d->numSMs * d->maxBlocksPerSM;
    if (cudaStreamCreateWithFlags(&d->ownStream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&d->ev0) != cudaSuccess || cudaEventCreate(&d->ev1) != cudaSuccess ||
        cudaMalloc((void**)&d->d_part, partCount * sizeof(double)) != cudaSuccess ||
        cudaMalloc((void**)&d->d_st, sizeof(InnerState)) != cudaSuccess ||
        cudaMalloc((void**)&d->d_drv, sizeof(DriverState)) != cudaSuccess ||
        cudaMalloc((void**)&d->d_chebC, sizeof(float) * 2 * CF_MAX_CHEB) != cudaSuccess ||
        cudaMalloc((void**)&d->d_sums, sizeof(double) * 8) != cudaSuccess ||
        cudaMalloc((void**)&d->d_census, sizeof(double) * 2) != cudaSuccess ||
        cudaMallocHost((void**)&d->h_st, sizeof(InnerState)) != cudaSuccess ||
        cudaMallocHost((void**)&d->h_drv, sizeof(DriverState)) != cudaSuccess ||
        cudaMallocHost((void**)&d->h_sums, sizeof(double) * 8) != cudaSuccess)
    {
        cudaGetLastError();
        cf_subdomain_destroy(d);
        return fail(CF_ERR_CUDA, "cf_subdomain_create: allocation failed");
    }
    d->stream = d->ownStream;
    cudaMemset(d->d_st, 0, sizeof(InnerState));
    cudaMemset(d->d_drv, 0, sizeof(DriverState));
    cudaMemset(d->d_part, 0, partCount * sizeof(double));
    *out = d;
    return CF_OK;
}

extern "C" int cf_subdomain_destroy(cf_subdomain* d)
{
    if (!d) return CF_OK;
    cudaSetDevice(d->device);
    if (d->stream) cudaStreamSynchronize(d->stream);
    free_topology(d);
    if (d->d_part) cudaFree(d->d_part);
    if (d->d_st) cudaFree(d->d_st);
    if (d->d_drv) cudaFree(d->d_drv);
    if (d->d_chebC) cudaFree(d->d_chebC);
    if (d->d_sums) cudaFree(d->d_sums);
    if (d->d_census) cudaFree(d->d_census);
    if (d->h_st) cudaFreeHost(d->h_st);
    if (d->h_drv) cudaFreeHost(d->h_drv);
    if (d->h_sums) cudaFreeHost(d->h_sums);
    if (d->ev0) cudaEventDestroy(d->ev0);
    if (d->ev1) cudaEventDestroy(d->ev1);
    if (d->ownStream) cudaStreamDestroy(d->ownStream);
    delete d;
    return CF_OK;
}

extern "C" int cf_subdomain_set_stream(cf_subdomain* d, void* stream)
{
    if (!d) return fail(CF_ERR_INVALID_ARG, "subdomain is NULL");
    d->stream = stream ? (cudaStream_t)stream : d->ownStream;
    return CF_OK;
}

extern "C" int cf_subdomain_set_topology(cf_subdomain* d, int32_t n, int32_t nf,
                                         const int32_t* low, const int32_t* upp,
                                         const int32_t* own, const int32_t* los,
                                         const int32_t* losS, int32_t nInterfaces,
                                         const int32_t* neighbour, const int32_t* nFaces,
                                         const int32_t* faceCells, int32_t reorder)
{
    if (!d) return fail(CF_ERR_INVALID_ARG, "subdomain is NULL");
    if (n <= 0 || nf < 0 || nInterfaces < 0)
        return fail(CF_ERR_INVALID_ARG, "nCells must be > 0, nFaces and nInterfaces >= 0");
    if ((nf > 0 && (!low || !upp || !los)) || !own || !losS ||
        (nInterfaces > 0 && (!neighbour || !nFaces || !faceCells)))
        return fail(CF_ERR_INVALID_ARG, "NULL addressing array");
    if (reorder < CF_REORDER_NONE || reorder > CF_REORDER_AUTO)
        return fail(CF_ERR_INVALID_ARG, "bad reorder mode");
    CF_TRY(check_addressing(n, nf, low, upp, own, los, losS));
    long long nH = 0;
    for (int p = 0; p < nInterfaces; ++p)
    {
        if (nFaces[p] < 0) return fail(CF_ERR_INVALID_ARG, "negative interface size");
        for (int q = 0; q < p; ++q)
            if (neighbour[q] == neighbour[p])
                return fail(CF_ERR_UNSUPPORTED, "one interface per neighbouring subdomain");
        nH += nFaces[p];
    }
    if (nH + n >= (1LL << 31) - 1024) return fail(CF_ERR_TOO_LARGE, "subdomain too large");
    for (long long h = 0; h < nH; ++h)
        if (faceCells[h] < 0 || faceCells[h] >= n)
            return fail(CF_ERR_BAD_ADDRESSING, "interface faceCells out of range");
    CF_CUDA(cudaSetDevice(d->device));
    CF_CUDA(cudaStreamSynchronize(d->stream));
    free_topology(d);
    d->n = n;
    d->nf = nf;
    d->nIf = nInterfaces;
    d->nH = (int)nH;
    d->nX = n + (int)nH;
    d->nbr.assign(neighbour, neighbour + nInterfaces);
    d->nFaces.assign(nFaces, nFaces + nInterfaces);
    d->haloOff.assign(nInterfaces + 1, 0);
    for (int p = 0; p < nInterfaces; ++p) d->haloOff[p + 1] = d->haloOff[p] + nFaces[p];
    // interface faces as extra row entries: CSR over cells in interface order
    std::vector<int32_t> xStart(n + 1, 0), xCol((size_t)std::max(nH, 1LL)),
        xFace((size_t)std::max(nH, 1LL));
    for (long long h = 0; h < nH; ++h) xStart[faceCells[h] + 1]++;
    for (int i = 0; i < n; ++i) xStart[i + 1] += xStart[i];
    {
        std::vector<int32_t> fill(xStart.begin(), xStart.end() - 1);
        for (long long h = 0; h < nH; ++h)
        {
            const int32_t k = fill[faceCells[h]]++;
            xCol[k] = n + (int32_t)h;
            xFace[k] = nf + (int32_t)h;
        }
    }
    const bool rcm = reorder == CF_REORDER_RCM || (reorder == CF_REORDER_AUTO && n > 65536);
    HostLayout L;
    CF_TRY(build_layout(n, nf, low, upp, own, los, losS, rcm, L, xStart.data(), xCol.data(),
                        xFace.data()));
    d->perm = L.perm;
    d->nslices = L.nslices;
    d->nnzp = L.nnzp;
    d->ellW = L.uniformW;
    std::vector<int32_t> iperm(n);
    for (int r = 0; r < n; ++r) iperm[L.perm[r]] = r;
    std::vector<int32_t> sendRow((size_t)std::max(nH, 1LL), 0);
    for (long long h = 0; h < nH; ++h) sendRow[h] = iperm[faceCells[h]];
    const size_t N = (size_t)n, NX = (size_t)d->nX, NE = (size_t)std::max(L.nnzp, 1LL);
    CF_TRY(sd_alloc(d, &d->d_sliceOff, (size_t)L.nslices + 1));
    CF_TRY(sd_alloc(d, &d->d_col, NE));
    CF_TRY(sd_alloc(d, &d->d_eface, NE));
    CF_TRY(sd_alloc(d, &d->d_perm, N));
    CF_TRY(sd_alloc(d, &d->d_sendRow, sendRow.size()));
    CF_TRY(sd_alloc(d, &d->d_val32, NE));
    CF_TRY(sd_alloc(d, &d->d_val64, NE));
    CF_TRY(sd_alloc(d, &d->d_valT64, NE));
    CF_TRY(sd_alloc(d, &d->d_upperX, (size_t)nf + (size_t)nH));
    CF_TRY(sd_alloc(d, &d->d_lowerX, (size_t)nf + (size_t)nH));
    CF_TRY(sd_alloc(d, &d->d_diagIn, N));
    CF_TRY(sd_alloc(d, &d->d_diag64, N));
    CF_TRY(sd_alloc(d, &d->d_u, N));
    CF_TRY(sd_alloc(d, &d->d_diag32, N));
    CF_TRY(sd_alloc(d, &d->d_rD32, N));
    CF_TRY(sd_alloc(d, &d->d_psi, NX));
    CF_TRY(sd_alloc(d, &d->d_b, N));
    CF_TRY(sd_alloc(d, &d->d_r64, N));
    CF_TRY(sd_alloc(d, &d->d_io64, N));
    CF_TRY(sd_alloc(d, &d->d_rA, N));
    CF_TRY(sd_alloc(d, &d->d_W0, NX));
    CF_TRY(sd_alloc(d, &d->d_W1, NX));
    CF_TRY(sd_alloc(d, &d->d_Z0, NX));
    CF_TRY(sd_alloc(d, &d->d_Z1, NX));
    CF_TRY(sd_alloc(d, &d->d_P, 2 * NX));
    CF_TRY(sd_alloc(d, &d->d_Q, N));
    CF_TRY(sd_alloc(d, &d->d_T, N));
    CF_TRY(sd_alloc(d, &d->d_D, 3 * N));
    CF_TRY(sd_alloc(d, &d->d_send32, (size_t)std::max(nH, 1LL)));
    CF_TRY(sd_alloc(d, &d->d_send64, (size_t)std::max(nH, 1LL)));
    CF_CUDA(cudaMallocHost((void**)&d->h_send, sizeof(double) * (size_t)std::max(nH, 1LL)));
    CF_CUDA(cudaMallocHost((void**)&d->h_recv, sizeof(double) * (size_t)std::max(nH, 1LL)));
    cudaStream_t s = d->stream;
    CF_CUDA(cudaMemcpyAsync(d->d_sliceOff, L.sliceOff.data(), sizeof(int32_t) * L.sliceOff.size(),
                            cudaMemcpyHostToDevice, s));
    CF_CUDA(cudaMemcpyAsync(d->d_col, L.col.data(), sizeof(int32_t) * L.col.size(),
                            cudaMemcpyHostToDevice, s));
    CF_CUDA(cudaMemcpyAsync(d->d_eface, L.eface.data(), sizeof(int32_t) * L.eface.size(),
                            cudaMemcpyHostToDevice, s));
    CF_CUDA(cudaMemcpyAsync(d->d_perm, L.perm.data(), sizeof(int32_t) * N, cudaMemcpyHostToDevice,
                            s));
    CF_CUDA(cudaMemcpyAsync(d->d_sendRow, sendRow.data(), sizeof(int32_t) * sendRow.size(),
                            cudaMemcpyHostToDevice, s));
    // halo tails start finite; every vector a kernel may read is defined
    CF_CUDA(cudaMemsetAsync(d->d_psi, 0, sizeof(double) * NX, s));
    for (float* v : {d->d_W0, d->d_W1, d->d_Z0, d->d_Z1})
        CF_CUDA(cudaMemsetAsync(v, 0, sizeof(float) * NX, s));
    CF_CUDA(cudaMemsetAsync(d->d_P, 0, sizeof(float) * 2 * NX, s));
    CF_CUDA(cudaMemsetAsync(d->d_D, 0, sizeof(float) * 3 * N, s));
    CF_CUDA(cudaMemsetAsync(d->d_upperX, 0, sizeof(double) * ((size_t)nf + nH), s));
    CF_CUDA(cudaMemsetAsync(d->d_lowerX, 0, sizeof(double) * ((size_t)nf + nH), s));
    CF_CUDA(cudaStreamSynchronize(s));
    d->val32Sym = -1;
    d->hasTopo = true;
    return CF_OK;
}

extern "C" int cf_subdomain_set_coeffs(cf_subdomain* d, const double* diag, const double* upper,
                                       const double* lower, const double* interfaceCoeffs)
{
    if (!d) return fail(CF_ERR_INVALID_ARG, "subdomain is NULL");
    if (!d->hasTopo) return fail(CF_ERR_NO_TOPOLOGY, "cf_subdomain_set_topology has not been called");
    if (!diag || (d->nf > 0 && !upper) || (d->nH > 0 && !interfaceCoeffs))
        return fail(CF_ERR_INVALID_ARG, "NULL coefficient array");
    CF_CUDA(cudaSetDevice(d->device));
    cudaStream_t s = d->stream;
    const int n = d->n, nf = d->nf, nH = d->nH;
    // interface entries carry -coeff (Amul subtracts coeff * psi_neighbour)
    std::vector<double> neg((size_t)std::max(nH, 1));
    for (int h = 0; h < nH; ++h) neg[h] = -interfaceCoeffs[h];
    CF_CUDA(cudaMemcpyAsync(d->d_diagIn, diag, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    if (nf > 0)
    {
        CF_CUDA(cudaMemcpyAsync(d->d_upperX, upper, sizeof(double) * nf, cudaMemcpyHostToDevice, s));
        CF_CUDA(cudaMemcpyAsync(d->d_lowerX, lower ? lower : upper, sizeof(double) * nf,
                                cudaMemcpyHostToDevice, s));
    }
    if (nH > 0)
    {
        CF_CUDA(cudaMemcpyAsync(d->d_upperX + nf, neg.data(), sizeof(double) * nH,
                                cudaMemcpyHostToDevice, s));
        CF_CUDA(cudaMemcpyAsync(d->d_lowerX + nf, neg.data(), sizeof(double) * nH,
                                cudaMemcpyHostToDevice, s));
    }
    d->hasLower = lower != nullptr;
    k_gather_f64<<<grid_of(d, (const void*)k_gather_f64, n), NT, 0, s>>>(n, d->d_perm, d->d_diagIn,
                                                                          d->d_diag64);
    CF_LAUNCH();
    CF_TRY(stage_vals_sd(d, d->hasLower ? 0 : 1));
    kc_sumA<MW><<<grid_of(d, (const void*)k_sumA<MW>, n), NT, 0, s>>>(
        sell_sd(d), d->d_diag64, d->d_u, d->d_census, &d->d_drv->ticket, d->d_part);
    CF_LAUNCH();
    CF_TRY(stage_diag32_sd(d, 0));
    CF_CUDA(cudaStreamSynchronize(s));   // the host copies above go out of scope
    d->hasCoeffs = true;
    return CF_OK;
}

extern "C" int cf_subdomain_solve(cf_subdomain* d, int32_t solver, double* psi,
                                  const double* source, const cf_options* opts,
                                  const cf_comm* comm, cf_performance* perf)
{
    if (!d || !psi || !source || !opts || !comm || !perf || !comm->allreduce || !comm->exchange)
        return fail(CF_ERR_INVALID_ARG, "NULL argument");
    if (!d->hasTopo) return fail(CF_ERR_NO_TOPOLOGY, "cf_subdomain_set_topology has not been called");
    if (!d->hasCoeffs) return fail(CF_ERR_NO_COEFFS, "cf_subdomain_set_coeffs has not been called");
    if (solver != CF_SOLVER_PCG && solver != CF_SOLVER_PBICGSTAB)
        return fail(CF_ERR_INVALID_ARG, "unknown solver");
    if (opts->preconditioner != CF_PRECOND_CHEBYSHEV)
        return fail(CF_ERR_UNSUPPORTED, "coupled solves use the Chebyshev-Jacobi preconditioner");
    if (opts->deflate < CF_DEFLATE_AUTO || opts->deflate > CF_DEFLATE_OFF || opts->maxRestarts < 0 ||
        !(opts->chebyshevRatio > 1.0))
        return fail(CF_ERR_INVALID_ARG, "bad options");
    CF_CUDA(cudaSetDevice(d->device));
    Ctx x{d, comm};
    const int rc = solve_sd(x, solver, psi, source, cudaMemcpyHostToDevice, opts, perf);
    if (rc != CF_OK && comm->abort) comm->abort(comm->user);
    return rc;
}

extern "C" int cf_subdomain_kernel_launches(const cf_subdomain* d, long long* count)
{
    if (!d || !count) return fail(CF_ERR_INVALID_ARG, "NULL argument");
    *count = d->launches;
    return CF_OK;
}

// ------------------------------------------------- subdomains of one process

namespace {

// Host-side rendezvous of the subdomains of one process (one thread each):
// kernels never wait on one another; the host threads meet at a barrier
// with a time limit, after which (or after an abort) every call fails.
struct LocalHub
{
    int nRanks = 0;
    int device = 0;
    std::mutex m;
    std::condition_variable cv;
    int arrived = 0;
    long long gen = 0;
    bool aborted = false;
    double timeoutSeconds = 120.0;
    std::vector<const void* const*> send;
    std::vector<const int32_t*> nbr, nFaces;
    std::vector<int> nIf;
    std::vector<std::vector<double>> vals;

    int barrier()
    {
        std::unique_lock<std::mutex> lk(m);
        if (aborted) return 1;
        const long long g = gen;
        if (++arrived == nRanks)
        {
            arrived = 0;
            ++gen;
            cv.notify_all();
            return 0;
        }
        const bool ok = cv.wait_for(lk, std::chrono::duration<double>(timeoutSeconds),
                                    [&] { return gen != g || aborted; });
        if (!ok || aborted)
        {
            aborted = true;
            cv.notify_all();
            return 1;
        }
        return 0;
    }
};

struct LocalRank
{
    LocalHub* hub;
    int rank;
};

int local_allreduce(void* user, double* values, int32_t count, int32_t op, void* stream)
{
    LocalRank* lr = (LocalRank*)user;
    LocalHub* h = lr->hub;
    cudaStream_t s = (cudaStream_t)stream;
    std::vector<double>& mine = h->vals[lr->rank];
    mine.assign(count, 0.0);
    if (cudaMemcpyAsync(mine.data(), values, sizeof(double) * count, cudaMemcpyDeviceToHost, s) !=
            cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return 2;
    if (h->barrier()) return 1;
    // every rank folds in rank order: identical results everywhere
    std::vector<double> out(count);
    for (int i = 0; i < count; ++i)
    {
        double a = h->vals[0][i];
        for (int r = 1; r < h->nRanks; ++r)
            a = op == 1 ? std::max(a, h->vals[r][i]) : a + h->vals[r][i];
        out[i] = a;
    }
    if (h->barrier()) return 1;
    if (cudaMemcpyAsync(values, out.data(), sizeof(double) * count, cudaMemcpyHostToDevice, s) !=
            cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return 2;
    return 0;
}

int local_exchange(void* user, int32_t nIf, const int32_t* nbr, const int32_t* nFaces,
                   int32_t elemBytes, const void* const* send, void* const* recv, void* stream)
{
    LocalRank* lr = (LocalRank*)user;
    LocalHub* h = lr->hub;
    const int a = lr->rank;
    cudaStream_t s = (cudaStream_t)stream;
    if (cudaStreamSynchronize(s) != cudaSuccess) return 2;   // send buffers complete
    h->send[a] = send;
    h->nbr[a] = nbr;
    h->nFaces[a] = nFaces;
    h->nIf[a] = nIf;
    if (h->barrier()) return 1;
    int rc = 0;
    for (int p = 0; p < nIf && rc == 0; ++p)
    {
        const int b = nbr[p];
        if (b < 0 || b >= h->nRanks)
        {
            rc = 3;
            break;
        }
        int q = -1;
        for (int k = 0; k < h->nIf[b]; ++k)
            if (h->nbr[b][k] == a) q = k;
        if (q < 0 || h->nFaces[b][q] != nFaces[p])
        {
            rc = 3;   // the neighbour has no matching interface
            break;
        }
        if (nFaces[p] > 0 &&
            cudaMemcpyAsync(recv[p], h->send[b][q], (size_t)nFaces[p] * elemBytes,
                            cudaMemcpyDefault, s) != cudaSuccess)
            rc = 2;
    }
    if (rc == 0 && cudaStreamSynchronize(s) != cudaSuccess) rc = 2;
    if (rc != 0)
    {
        std::lock_guard<std::mutex> lk(h->m);
        h->aborted = true;
        h->cv.notify_all();
        return rc;
    }
    if (h->barrier()) return 1;   // nobody reuses a send buffer before all have read it
    return 0;
}

void local_abort(void* user)
{
    LocalHub* h = ((LocalRank*)user)->hub;
    std::lock_guard<std::mutex> lk(h->m);
    h->aborted = true;
    h->cv.notify_all();
}

}  // namespace

extern "C" int cf_comm_local_create(int32_t nRanks, double timeoutSeconds, cf_comm* comms)
{
    if (nRanks < 1 || nRanks > 1024 || !comms || !(timeoutSeconds > 0.0))
        return fail(CF_ERR_INVALID_ARG, "cf_comm_local_create: bad arguments");
    LocalHub* h = new LocalHub();
    h->nRanks = nRanks;
    h->timeoutSeconds = timeoutSeconds;
    h->send.assign(nRanks, nullptr);
    h->nbr.assign(nRanks, nullptr);
    h->nFaces.assign(nRanks, nullptr);
    h->nIf.assign(nRanks, 0);
    h->vals.assign(nRanks, {});
    for (int r = 0; r < nRanks; ++r)
    {
        comms[r].user = new LocalRank{h, r};
        comms[r].allreduce = local_allreduce;
        comms[r].exchange = local_exchange;
        comms[r].abort = local_abort;
        comms[r].hostBuffers = 0;
    }
    return CF_OK;
}

extern "C" int cf_comm_local_destroy(int32_t nRanks, cf_comm* comms)
{
    if (nRanks < 1 || !comms) return fail(CF_ERR_INVALID_ARG, "bad arguments");
    LocalHub* h = ((LocalRank*)comms[0].user)->hub;
    for (int r = 0; r < nRanks; ++r)
    {
        delete (LocalRank*)comms[r].user;
        comms[r].user = nullptr;
    }
    delete h;
    return CF_OK;
}
