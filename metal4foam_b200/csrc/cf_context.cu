// cf_context.cu -- host side of the C ABI (include/cudafoam.h): context,
// topology (validation, internal ordering, SELL-32 layout), coefficient
// staging, the inner FP32 solves driven on the device by CUDA-graph
// conditional WHILE nodes, and the FP64 refinement driver.
//
// Reference counterparts: metalFoamBackend::{Impl::init, setTopology,
// setCoeffs, pcg, bicgstab, delta} (src/metal4Foam/backend/metalFoamBackend.C)
// and metalFoamSolver::solveImpl (src/metal4Foam/solvers/metalFoamSolver.C).
#include "cudafoam.h"
#include "cf_internal.cuh"
#include "cf_kernels.cuh"
#include "cf_host.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <utility>
#include <vector>

using namespace cf;

namespace cf {

thread_local std::string g_err;

int fail(int code, const std::string& msg)
{
    g_err = msg;
    return code;
}

double wall_now()
{
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

}  // namespace cf

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

// ------------------------------------------------------------------ helpers

namespace {

template <class T>
int dalloc(cf_context* c, T** p, size_t count)
{
    *p = nullptr;
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc((void**)p, count * sizeof(T));
    if (e != cudaSuccess)
        return fail(CF_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    c->topoAllocs.push_back((void*)*p);
    return CF_OK;
}

void free_topology(cf_context* c)
{
    for (cf_context* k : c->clones) cf_context_destroy(k);
    c->clones.clear();
    cf_multi_release(c);
    amg_release(c);
    for (auto& kv : c->graphs) cudaGraphExecDestroy(kv.second);
    c->graphs.clear();
    for (void* p : c->topoAllocs) cudaFree(p);
    c->topoAllocs.clear();
    c->lduReady = false;
    c->d_own = c->d_losS = c->d_los = c->d_uppI = c->d_lowI = nullptr;
    c->d_face32 = nullptr;
    c->hasTopo = false;
    c->hasCoeffs = false;
    c->n = c->nf = 0;
    c->lastLow = c->lastUpp = nullptr;
    c->d_col16 = nullptr;
    c->d_pcol16 = nullptr;
    c->d_pval32 = nullptr;
}

// Validate the five lduAddressing arrays (the bounds check the reference
// lacks: SECURITY.md names OOB reads on malformed matrices as its risk).
int validate_addressing(int32_t n, int32_t nf, const int32_t* low, const int32_t* upp,
                        const int32_t* own, const int32_t* los, const int32_t* losS)
{
    for (int32_t f = 0; f < nf; ++f)
    {
        if (low[f] < 0 || upp[f] >= n || low[f] >= upp[f])
            return fail(CF_ERR_BAD_ADDRESSING, "face " + std::to_string(f) +
                                                   ": owner/neighbour out of range or owner >= neighbour");
        if (f > 0 && (low[f] < low[f - 1] || (low[f] == low[f - 1] && upp[f] <= upp[f - 1])))
            return fail(CF_ERR_BAD_ADDRESSING, "faces not sorted by owner then neighbour at face " +
                                                   std::to_string(f));
    }
    if (own[0] != 0 || own[n] != nf || losS[0] != 0 || losS[n] != nf)
        return fail(CF_ERR_BAD_ADDRESSING, "ownerStart/losortStart must start at 0 and end at nFaces");
    for (int32_t i = 0; i < n; ++i)
    {
        if (own[i + 1] < own[i] || losS[i + 1] < losS[i])
            return fail(CF_ERR_BAD_ADDRESSING, "ownerStart/losortStart not monotone at cell " +
                                                   std::to_string(i));
        for (int32_t f = own[i]; f < own[i + 1]; ++f)
            if (low[f] != i)
                return fail(CF_ERR_BAD_ADDRESSING, "ownerStart inconsistent with lowerAddr at cell " +
                                                       std::to_string(i));
        for (int32_t k = losS[i]; k < losS[i + 1]; ++k)
        {
            const int32_t f = los[k];
            if (f < 0 || f >= nf || upp[f] != i || (k > losS[i] && f <= los[k - 1]))
                return fail(CF_ERR_BAD_ADDRESSING, "losort inconsistent with upperAddr at cell " +
                                                       std::to_string(i));
        }
    }
    return CF_OK;
}

// Reverse Cuthill-McKee ordering of the cell graph (pseudo-peripheral start
// per connected component, neighbours visited by ascending degree).  Makes
// the x-gathers of a warp's 32 rows hit a few cache lines even when the
// mesh's own numbering is scattered.
void rcm_order(int32_t n, const int32_t* low, const int32_t* upp, const int32_t* own,
               const int32_t* los, const int32_t* losS, std::vector<int32_t>& perm)
{
    std::vector<int32_t> deg(n);
    for (int32_t i = 0; i < n; ++i) deg[i] = (own[i + 1] - own[i]) + (losS[i + 1] - losS[i]);
    auto for_nbrs = [&](int32_t v, auto&& fn) {
        for (int32_t f = own[v]; f < own[v + 1]; ++f) fn(upp[f]);
        for (int32_t k = losS[v]; k < losS[v + 1]; ++k) fn(low[los[k]]);
    };
    std::vector<int32_t> mark(n, -1);  // search stamp
    std::vector<char> done(n, 0);
    std::vector<int32_t> queue;
    queue.reserve(n);
    perm.clear();
    perm.reserve(n);
    int32_t stamp = 0;
    std::vector<int32_t> nb;
    for (int32_t s0 = 0; s0 < n; ++s0)
    {
        if (done[s0]) continue;
        // George-Liu pseudo-peripheral node search
        int32_t start = s0;
        int32_t ecc = -1;
        for (int pass = 0; pass < 6; ++pass)
        {
            ++stamp;
            queue.clear();
            queue.push_back(start);
            mark[start] = stamp;
            size_t head = 0;
            int32_t levels = 0;
            size_t levelBegin = 0;
            while (head < queue.size())
            {
                const size_t levelEnd = queue.size();
                levelBegin = head;
                while (head < levelEnd)
                {
                    const int32_t v = queue[head++];
                    for_nbrs(v, [&](int32_t w) {
                        if (mark[w] != stamp)
                        {
                            mark[w] = stamp;
                            queue.push_back(w);
                        }
                    });
                }
                ++levels;
            }
            int32_t best = queue[levelBegin];
            for (size_t q = levelBegin; q < queue.size(); ++q)
                if (deg[queue[q]] < deg[best]) best = queue[q];
            if (levels <= ecc) break;
            ecc = levels;
            if (best == start) break;
            start = best;
        }
        // Cuthill-McKee from start
        size_t head = perm.size();
        perm.push_back(start);
        done[start] = 1;
        while (head < perm.size())
        {
            const int32_t v = perm[head++];
            nb.clear();
            for_nbrs(v, [&](int32_t w) {
                if (!done[w])
                {
                    done[w] = 1;
                    nb.push_back(w);
                }
            });
            std::stable_sort(nb.begin(), nb.end(),
                             [&](int32_t a, int32_t b) { return deg[a] < deg[b]; });
            perm.insert(perm.end(), nb.begin(), nb.end());
        }
    }
    std::reverse(perm.begin(), perm.end());
}

}  // namespace

namespace cf {

int check_addressing(int32_t n, int32_t nf, const int32_t* low, const int32_t* upp,
                     const int32_t* own, const int32_t* los, const int32_t* losS)
{
    return validate_addressing(n, nf, low, upp, own, los, losS);
}

// Internal ordering + SELL-32 layout of one mesh on the host.
int build_layout(int32_t n, int32_t nf, const int32_t* low, const int32_t* upp,
                 const int32_t* own, const int32_t* los, const int32_t* losS, bool rcm,
                 HostLayout& L, const int32_t* xStart, const int32_t* xCol,
                 const int32_t* xFace)
{
    (void)nf;
    // extra entries of cell i (xStart[i] .. xStart[i+1]) follow its losort
    // faces; their columns are already internal (not relabelled)
    auto nExtra = [&](int32_t i) { return xStart ? xStart[i + 1] - xStart[i] : 0; };
    std::vector<int32_t>& perm = L.perm;
    perm.clear();
    if (rcm) rcm_order(n, low, upp, own, los, losS, perm);
    if ((int32_t)perm.size() != n)
    {
        perm.resize(n);
        for (int32_t i = 0; i < n; ++i) perm[i] = i;
    }
    std::vector<int32_t> iperm(n);
    for (int32_t r = 0; r < n; ++r) iperm[perm[r]] = r;

    const int32_t nslices = (n + SLICE - 1) / SLICE;
    L.sliceOff.assign(nslices + 1, 0);
    std::vector<int32_t> sw(nslices, 0);
    long long nnzSell = 0;
    int32_t wmax = 0;
    for (int32_t s = 0; s < nslices; ++s)
    {
        int32_t w = 0;
        for (int32_t l = 0; l < SLICE; ++l)
        {
            const int32_t r = s * SLICE + l;
            if (r >= n) break;
            const int32_t i = perm[r];
            w = std::max(w, (own[i + 1] - own[i]) + (losS[i + 1] - losS[i]) + nExtra(i));
        }
        sw[s] = w;
        nnzSell += (long long)w * SLICE;
        wmax = std::max(wmax, w);
    }
    // one width for every slice when that pads at most 1/16 more entries:
    // slice s then starts at 32 s W and the kernels need no sliceOff load
    L.uniformW = 0;
    if (wmax > 0 && (long long)nslices * SLICE * wmax <= nnzSell + nnzSell / 16)
    {
        L.uniformW = wmax;
        for (int32_t s = 0; s < nslices; ++s) sw[s] = wmax;
    }
    long long nnzp = 0;
    for (int32_t s = 0; s < nslices; ++s)
    {
        const int32_t w = sw[s];
        nnzp += (long long)w * SLICE;
        if (nnzp >= (1LL << 31) - 64)
            return fail(CF_ERR_TOO_LARGE, "matrix too large for 32-bit entry offsets");
        L.sliceOff[s + 1] = (int32_t)nnzp;
    }
    L.col.assign((size_t)std::max(nnzp, 1LL), -1);
    L.eface.assign((size_t)std::max(nnzp, 1LL), -1);
    int32_t maxw = 0;
    for (int32_t r = 0; r < n; ++r)
    {
        const int32_t i = perm[r];
        const int32_t s = r / SLICE;
        const int32_t lane = r % SLICE;
        int32_t k = 0;
        for (int32_t f = own[i]; f < own[i + 1]; ++f, ++k)
        {
            const size_t e = (size_t)L.sliceOff[s] + (size_t)SLICE * k + lane;
            L.col[e] = iperm[upp[f]];
            L.eface[e] = f;
        }
        for (int32_t q = losS[i]; q < losS[i + 1]; ++q, ++k)
        {
            const int32_t f = los[q];
            const size_t e = (size_t)L.sliceOff[s] + (size_t)SLICE * k + lane;
            L.col[e] = (int32_t)((uint32_t)iperm[low[f]] | 0x80000000u);
            L.eface[e] = f;
        }
        for (int32_t x = 0; x < nExtra(i); ++x, ++k)
        {
            const size_t e = (size_t)L.sliceOff[s] + (size_t)SLICE * k + lane;
            L.col[e] = xCol[xStart[i] + x];
            L.eface[e] = xFace[xStart[i] + x];
        }
        maxw = std::max(maxw, k);
    }
    L.nslices = nslices;
    L.nnzp = nnzp;
    L.maxw = maxw;
    return CF_OK;
}

int grid_for(cf_context* c, const void* fn, long long work)
{
    int occ = 0;
    auto it = c->occ.find(fn);
    if (it == c->occ.end())
    {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, NT, 0) != cudaSuccess) occ = 1;
        occ = std::max(1, std::min(occ, c->maxBlocksPerSM));
        c->occ[fn] = occ;
    }
    else
    {
        occ = it->second;
    }
    const long long cap = (long long)c->numSMs * occ;
    const long long need = (work + NT - 1) / NT;
    return (int)std::max(1LL, std::min(cap, need));
}

DevSell sell_of(const cf_context* c)
{
    DevSell A;
    A.n = c->n;
    A.nslices = c->nslices;
    A.sliceOff = c->d_sliceOff;
    A.col = c->d_col;
    A.val = c->d_val32;
    A.val64 = c->d_val64;
    A.col16 = c->cfgIndexBits == 16 ? c->d_col16 : nullptr;
    if (A.col16 && c->d_pcol16 && c->ellW > 0)
    {
        A.pcol16 = c->d_pcol16;
        A.pval = c->d_pval32;
    }
    A.ellW = c->ellW;
    return A;
}

PcgBufs pcg_bufs(const cf_context* c)
{
    PcgBufs B;
    B.rA = c->d_rA;
    B.W0 = c->d_W0;
    B.W1 = c->d_W1;
    B.Z0 = c->d_Z0;
    B.Z1 = c->d_Z1;
    B.P = c->d_P;
    B.Q = c->d_Q;
    B.D = c->d_D;
    B.diag = c->d_diag32;
    B.rD = c->d_rD32;
    B.chebC = c->d_chebC;
    B.r64 = c->d_r64;
    B.n = c->n;
    return B;
}

BicgBufs bicg_bufs(const cf_context* c)
{
    BicgBufs B;
    B.rA = c->d_rA;
    B.rA0 = c->d_W0;
    B.P = c->d_P;
    B.yA = c->d_W1;
    B.AyA = c->d_Q;
    B.sA = c->d_Z0;
    B.zA = c->d_Z1;
    B.tA = c->d_T;
    B.D = c->d_D;
    B.diag = c->d_diag32;
    B.rD = c->d_rD32;
    B.r64 = c->d_r64;
    B.n = c->n;
    return B;
}

}  // namespace cf

// ------------------------------------------------------------------ library

extern "C" int cf_abi_version(void) { return CF_ABI_VERSION; }

extern "C" const char* cf_last_error(void) { return g_err.c_str(); }

extern "C" void cf_options_default(cf_options* o)
{
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->tolerance = 1e-6;
    o->relTol = 0.0;
    o->maxIter = 1000;
    o->minIter = 0;
    o->maxRestarts = 8;
    o->iterationsPerSync = 1;
    o->deflate = CF_DEFLATE_AUTO;
    o->chebyshevOrder = 8;
    o->chebyshevRatio = 30.0;
    o->profile = 0;
    o->verbose = 0;
    o->graph = 1;
    o->preconditioner = CF_PRECOND_CHEBYSHEV;
    o->nSweeps = 3;
    o->nCellsInCoarsestLevel = 128;
    o->scaleCorrection = 1.8;
    o->smootherRatio = 8.0;
}

extern "C" int cf_context_create(cf_context** out, int32_t device)
{
    if (!out) return fail(CF_ERR_INVALID_ARG, "out is NULL");
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
    {
        cudaGetLastError();
        return fail(CF_ERR_NO_DEVICE, "cudaFoam: no CUDA device available");
    }
    if (device < 0 || device >= count)
        return fail(CF_ERR_INVALID_ARG, "device index out of range");
    cudaDeviceProp prop;
    CF_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10)
        return fail(CF_ERR_NO_DEVICE, std::string("cudaFoam: ") + prop.name +
                                          " is not an sm_100 (B200-class) device");
    CF_CUDA(cudaSetDevice(device));
    cf_context* c = new cf_context();
    c->device = device;
    c->numSMs = prop.multiProcessorCount;
    c->maxBlocksPerSM = std::max(1, prop.maxThreadsPerMultiProcessor / NT);
    c->maxCtasPerSM = std::max(c->maxBlocksPerSM, prop.maxBlocksPerMultiProcessor);
    c->coopLaunch = prop.cooperativeLaunch != 0;
    c->l2Bytes = prop.l2CacheSize;
    cudaError_t e = cudaStreamCreateWithFlags(&c->ownStream, cudaStreamNonBlocking);
    if (e != cudaSuccess)
    {
        delete c;
        return fail(CF_ERR_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
    }
    c->stream = c->ownStream;
    // reduction partials: NPART values for every block any launch shape can
    // keep resident (variant grids of 128-thread blocks exceed maxBlocksPerSM)
    const size_t partCount = (size_t)NPART * c->numSMs * c->maxCtasPerSM;
    if (cudaMalloc((void**)&c->d_part, partCount * sizeof(double)) != cudaSuccess ||
        cudaMalloc((void**)&c->d_st, sizeof(InnerState)) != cudaSuccess ||
        cudaMalloc((void**)&c->d_drv, sizeof(DriverState)) != cudaSuccess ||
        cudaMalloc((void**)&c->d_chebC, sizeof(float) * 2 * CF_MAX_CHEB) != cudaSuccess ||
        cudaMalloc((void**)&c->d_scratch64, sizeof(double) * 4) != cudaSuccess ||
        cudaMalloc((void**)&c->d_bar, sizeof(unsigned int) * 4) != cudaSuccess ||
        cudaMallocHost((void**)&c->h_st, sizeof(InnerState)) != cudaSuccess ||
        cudaMallocHost((void**)&c->h_drv, sizeof(DriverState)) != cudaSuccess)
    {
        cudaGetLastError();
        cf_context_destroy(c);
        return fail(CF_ERR_CUDA, "cudaFoam: allocation of context state failed");
    }
    cudaMemset(c->d_st, 0, sizeof(InnerState));
    cudaMemset(c->d_drv, 0, sizeof(DriverState));
    cudaMemset(c->d_scratch64, 0, sizeof(double) * 4);
    cudaEventCreate(&c->ev0);
    cudaEventCreate(&c->ev1);
    cudaEventCreate(&c->ev2);
    cudaEventCreate(&c->ev3);
    c->good = true;
    char buf[512];
    std::snprintf(buf, sizeof(buf), "cudaFoam: %s (sm_%d%d, %d SMs, %.0f MB L2)", prop.name,
                  prop.major, prop.minor, prop.multiProcessorCount, prop.l2CacheSize / 1048576.0);
    c->description = buf;
    *out = c;
    return CF_OK;
}

extern "C" int cf_context_destroy(cf_context* c)
{
    if (!c) return CF_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    free_topology(c);
    if (c->d_part) cudaFree(c->d_part);
    if (c->d_st) cudaFree(c->d_st);
    if (c->d_drv) cudaFree(c->d_drv);
    if (c->d_chebC) cudaFree(c->d_chebC);
    if (c->d_scratch64) cudaFree(c->d_scratch64);
    if (c->d_bar) cudaFree(c->d_bar);
    if (c->h_st) cudaFreeHost(c->h_st);
    if (c->h_drv) cudaFreeHost(c->h_drv);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->ev2) cudaEventDestroy(c->ev2);
    if (c->ev3) cudaEventDestroy(c->ev3);
    if (c->ownStream) cudaStreamDestroy(c->ownStream);
    delete c;
    return CF_OK;
}

extern "C" int cf_context_good(const cf_context* c) { return c && c->good ? 1 : 0; }

extern "C" const char* cf_context_description(const cf_context* c)
{
    return c ? c->description.c_str() : "cudaFoam: no context";
}

extern "C" int cf_context_set_stream(cf_context* c, void* stream)
{
    if (!c) return fail(CF_ERR_INVALID_ARG, "context is NULL");
    c->stream = stream ? (cudaStream_t)stream : c->ownStream;
    return CF_OK;
}

extern "C" int cf_context_set_reorder(cf_context* c, int32_t mode)
{
    if (!c || mode < CF_REORDER_NONE || mode > CF_REORDER_AUTO)
        return fail(CF_ERR_INVALID_ARG, "bad reorder mode");
    c->reorderMode = mode;
    return CF_OK;
}

extern "C" int cf_context_set_wait_limit(cf_context* c, int64_t polls)
{
    if (!c || polls < 0) return fail(CF_ERR_INVALID_ARG, "bad wait limit");
    c->waitPolls = polls == 0 ? (1LL << 24) : (long long)polls;
    return CF_OK;
}

extern "C" int cf_context_kernel_launches(const cf_context* c, long long* count)
{
    if (!c || !count) return fail(CF_ERR_INVALID_ARG, "NULL argument");
    *count = c->launches;
    return CF_OK;
}

// ------------------------------------------------------------------ topology

extern "C" int cf_set_topology(cf_context* c, int32_t n, int32_t nf, const int32_t* low,
                               const int32_t* upp, const int32_t* own, const int32_t* los,
                               const int32_t* losS)
{
    if (!c) return fail(CF_ERR_INVALID_ARG, "context is NULL");
    if (n <= 0 || nf < 0) return fail(CF_ERR_INVALID_ARG, "nCells must be > 0 and nFaces >= 0");
    if ((nf > 0 && (!low || !upp || !los)) || !own || !losS)
        return fail(CF_ERR_INVALID_ARG, "NULL addressing array");
    CF_CUDA(cudaSetDevice(c->device));
    // cache on identity, like metalFoamBackend.C:469-477
    if (c->hasTopo && c->n == n && c->nf == nf && c->lastLow == low && c->lastUpp == upp &&
        c->reorderMode == c->topoReorderMode)
        return CF_OK;
    CF_TRY(validate_addressing(n, nf, low, upp, own, los, losS));
    CF_CUDA(cudaStreamSynchronize(c->stream));
    free_topology(c);

    const bool rcm = c->reorderMode == CF_REORDER_RCM ||
                     (c->reorderMode == CF_REORDER_AUTO && n > 65536);
    HostLayout L;
    CF_TRY(build_layout(n, nf, low, upp, own, los, losS, rcm, L));
    std::vector<int32_t>& perm = L.perm;
    std::vector<int32_t>& sliceOff = L.sliceOff;
    std::vector<int32_t>& col = L.col;
    std::vector<int32_t>& eface = L.eface;
    const int32_t nslices = L.nslices;
    const long long nnzp = L.nnzp;
    const int32_t maxw = L.maxw;

    c->n = n;
    c->nf = nf;
    c->nslices = nslices;
    c->nnzp = nnzp;
    c->maxRowLen = maxw;
    c->ellW = L.uniformW;
    c->perm = perm;
    c->identityPerm = !rcm;
    const size_t N = (size_t)n;
    CF_TRY(dalloc(c, &c->d_sliceOff, nslices + 1));
    CF_TRY(dalloc(c, &c->d_col, (size_t)std::max(nnzp, 1LL)));
    CF_TRY(dalloc(c, &c->d_eface, (size_t)std::max(nnzp, 1LL)));
    CF_TRY(dalloc(c, &c->d_perm, N));
    CF_TRY(dalloc(c, &c->d_low, (size_t)std::max(nf, 1)));
    CF_TRY(dalloc(c, &c->d_upp, (size_t)std::max(nf, 1)));
    CF_TRY(dalloc(c, &c->d_val32, (size_t)std::max(nnzp, 1LL)));
    CF_TRY(dalloc(c, &c->d_val64, (size_t)std::max(nnzp, 1LL)));
    CF_TRY(dalloc(c, &c->d_valT64, (size_t)std::max(nnzp, 1LL)));
    CF_TRY(dalloc(c, &c->d_diagIn, N));
    CF_TRY(dalloc(c, &c->d_upper, (size_t)std::max(nf, 1)));
    CF_TRY(dalloc(c, &c->d_lower, (size_t)std::max(nf, 1)));
    CF_TRY(dalloc(c, &c->d_diag64, N));
    CF_TRY(dalloc(c, &c->d_u, N));
    CF_TRY(dalloc(c, &c->d_diag32, N));
    CF_TRY(dalloc(c, &c->d_rD32, N));
    CF_TRY(dalloc(c, &c->d_psi, N));
    CF_TRY(dalloc(c, &c->d_b, N));
    CF_TRY(dalloc(c, &c->d_r64, N));
    CF_TRY(dalloc(c, &c->d_io64, N));
    CF_TRY(dalloc(c, &c->d_io64b, N));
    CF_TRY(dalloc(c, &c->d_r0, N));
    CF_TRY(dalloc(c, &c->d_gU, (size_t)std::max(nf, 1)));
    CF_TRY(dalloc(c, &c->d_gL, (size_t)std::max(nf, 1)));
    CF_TRY(dalloc(c, &c->d_gD, N));
    c->hasResidual = false;
    c->transposed = false;
    CF_TRY(dalloc(c, &c->d_rA, N));
    CF_TRY(dalloc(c, &c->d_W0, N));
    CF_TRY(dalloc(c, &c->d_W1, N));
    CF_TRY(dalloc(c, &c->d_Z0, N));
    CF_TRY(dalloc(c, &c->d_Z1, N));
    CF_TRY(dalloc(c, &c->d_P, 2 * N));
    CF_TRY(dalloc(c, &c->d_Q, 2 * N));   // PCG: q; BiCGStab: A yA ping-pong
    CF_TRY(dalloc(c, &c->d_T, N));
    CF_TRY(dalloc(c, &c->d_D, 3 * N));
    CF_TRY(dalloc(c, &c->d_io32, N));
    CF_TRY(dalloc(c, &c->d_io32b, N));
    CF_TRY(dalloc(c, &c->d_io32c, N));
    CF_CUDA(cudaMemcpyAsync(c->d_sliceOff, sliceOff.data(), sizeof(int32_t) * (nslices + 1),
                            cudaMemcpyHostToDevice, c->stream));
    CF_CUDA(cudaMemcpyAsync(c->d_col, col.data(), sizeof(int32_t) * col.size(),
                            cudaMemcpyHostToDevice, c->stream));
    CF_CUDA(cudaMemcpyAsync(c->d_eface, eface.data(), sizeof(int32_t) * eface.size(),
                            cudaMemcpyHostToDevice, c->stream));
    CF_CUDA(cudaMemcpyAsync(c->d_perm, perm.data(), sizeof(int32_t) * N, cudaMemcpyHostToDevice,
                            c->stream));
    if (nf > 0)
    {
        CF_CUDA(cudaMemcpyAsync(c->d_low, low, sizeof(int32_t) * nf, cudaMemcpyHostToDevice,
                                c->stream));
        CF_CUDA(cudaMemcpyAsync(c->d_upp, upp, sizeof(int32_t) * nf, cudaMemcpyHostToDevice,
                                c->stream));
    }
    // compact column stream (row-relative 16-bit offsets) when every column
    // lies within 32767 rows of its row (the host copy lives until the
    // synchronisation below)
    std::vector<short> col16((size_t)std::max(nnzp, 1LL), COL16_PAD);
    std::vector<short> pcol16;
    {
        bool fits = true;
        for (int32_t sl = 0; sl < nslices && fits; ++sl)
        {
            const int32_t b0 = sliceOff[sl];
            const int32_t w = (sliceOff[sl + 1] - b0) / SLICE;
            for (int32_t k = 0; k < w && fits; ++k)
                for (int32_t l = 0; l < SLICE; ++l)
                {
                    const int32_t e = b0 + SLICE * k + l;
                    if (col[e] == -1) continue;
                    const long long off = (long long)(col[e] & 0x7fffffff) - (long long)(sl * SLICE + l);
                    if (off < -32767 || off > 32767)
                    {
                        fits = false;
                        break;
                    }
                    col16[e] = (short)off;
                }
        }
        if (fits)
        {
            CF_TRY(dalloc(c, &c->d_col16, col16.size()));
            CF_CUDA(cudaMemcpyAsync(c->d_col16, col16.data(), sizeof(short) * col16.size(),
                                    cudaMemcpyHostToDevice, c->stream));
            // the same stream in the paired order, with a paired copy of the
            // FP32 values (staged with them), when every slice has one width
            // with paired kernels
            if (L.uniformW >= PAIR_MIN_W && L.uniformW <= PAIR_MAX_W)
            {
                const int W = L.uniformW;
                const long long sw = (long long)SLICE * W;
                pcol16.assign(col16.size(), COL16_PAD);
                for (long long e = 0; e < nnzp; ++e)
                {
                    const long long sl = e / sw;
                    const int rem = (int)(e - sl * sw);
                    pcol16[pair_index(sl * sw, W, rem / SLICE, rem % SLICE)] = col16[e];
                }
                CF_TRY(dalloc(c, &c->d_pcol16, pcol16.size()));
                CF_TRY(dalloc(c, &c->d_pval32, pcol16.size()));
                CF_CUDA(cudaMemcpyAsync(c->d_pcol16, pcol16.data(),
                                        sizeof(short) * pcol16.size(), cudaMemcpyHostToDevice,
                                        c->stream));
            }
        }
    }
    // locality of the cluster PCG's row split (cf_cluster.cu): the share of
    // entries whose column belongs to another CTA
    {
        c->clusterShift = cluster_shift(n);
        long long entries = 0, remote = 0;
        for (int32_t sl = 0; sl < nslices; ++sl)
        {
            const int32_t b0 = sliceOff[sl];
            const int32_t w = (sliceOff[sl + 1] - b0) / SLICE;
            for (int32_t k = 0; k < w; ++k)
                for (int32_t l = 0; l < SLICE; ++l)
                {
                    const int32_t cc = col[(size_t)b0 + SLICE * k + l];
                    if (cc == -1) continue;
                    ++entries;
                    const int32_t row = sl * SLICE + l;
                    if (((cc & 0x7fffffff) >> c->clusterShift) != (row >> c->clusterShift)) ++remote;
                }
        }
        c->clusterRemote = entries ? (double)remote / (double)entries : 0.0;
    }
    CF_CUDA(cudaMemsetAsync(c->d_D, 0, sizeof(float) * 3 * N, c->stream));
    CF_CUDA(cudaMemsetAsync(c->d_r64, 0, sizeof(double) * N, c->stream));
    CF_CUDA(cudaStreamSynchronize(c->stream));
    c->hasTopo = true;
    c->lastLow = low;
    c->lastUpp = upp;
    c->topoReorderMode = c->reorderMode;
    return CF_OK;
}

// ------------------------------------------------------------------ coefficients

namespace cf {

int stage_vals(cf_context* c, int sym32)
{
    // A^T in LDU form is A with upper and lower exchanged
    const double* up = c->d_upper;
    const double* lo = c->hasLower ? c->d_lower : c->d_upper;
    if (c->transposed) std::swap(up, lo);
    const int g = grid_for(c, (const void*)k_stage_vals, c->nnzp);
    k_stage_vals<<<g, NT, 0, c->stream>>>(c->nnzp, c->d_col, c->d_eface, up, lo, sym32,
                                          c->d_val32, c->d_val64, c->d_valT64);
    CF_LAUNCH();
    if (c->d_pval32)
    {
        k_pair_vals<<<grid_for(c, (const void*)k_pair_vals, c->nnzp), NT, 0, c->stream>>>(
            c->nnzp, c->ellW, c->d_val32, c->d_pval32);
        CF_LAUNCH();
    }
    c->val32Sym = sym32;
    if (c->lduReady) CF_TRY(stage_face32(c, up, lo, sym32));
    return CF_OK;
}

// u = A 1 (of the staged operator) and the deflation census
int stage_rowsums(cf_context* c)
{
    auto fn = k_sumA<MAXW_UNROLL>;
    const int g = grid_for(c, (const void*)fn, c->n);
    fn<<<g, NT, 0, c->stream>>>(sell_of(c), c->d_diag64, c->d_u, c->d_drv, c->d_part);
    CF_LAUNCH();
    return CF_OK;
}

int stage_diag32(cf_context* c, int deflate)
{
    const int g = grid_for(c, (const void*)k_stage_diag32, c->n);
    k_stage_diag32<<<g, NT, 0, c->stream>>>(c->n, c->d_diag64, c->d_u, deflate, c->d_diag32,
                                            c->d_rD32);
    CF_LAUNCH();
    return CF_OK;
}

int stage_coeffs_from_device(cf_context* c)
{
    // internal-order FP64 diagonal, SELL values, sumA census, FP32 diag
    {
        const int g = grid_for(c, (const void*)k_gather_f64, c->n);
        k_gather_f64<<<g, NT, 0, c->stream>>>(c->n, c->d_perm, c->d_diagIn, c->d_diag64);
        CF_LAUNCH();
    }
    CF_TRY(stage_vals(c, c->hasLower ? 0 : 1));
    CF_TRY(stage_rowsums(c));
    CF_TRY(stage_diag32(c, 0));
    c->hasCoeffs = true;
    return CF_OK;
}

}  // namespace cf

namespace cf {

int context_clone_matrix(cf_context* src, cf_context** out)
{
    *out = nullptr;
    cf_context* c = nullptr;
    CF_TRY(cf_context_create(&c, src->device));
    struct Guard
    {
        cf_context* c;
        ~Guard()
        {
            if (c) cf_context_destroy(c);
        }
    } guard{c};
    c->reorderMode = src->reorderMode;
    c->topoReorderMode = src->topoReorderMode;
    c->n = src->n;
    c->nf = src->nf;
    c->nslices = src->nslices;
    c->nnzp = src->nnzp;
    c->maxRowLen = src->maxRowLen;
    c->ellW = src->ellW;
    c->perm = src->perm;
    c->identityPerm = src->identityPerm;
    c->clusterShift = src->clusterShift;
    c->clusterRemote = src->clusterRemote;
    // vectors of its own (the FP32 diagonal included: every solve stages it);
    // only cf_solve[_device] runs on a clone, so it has no face-gradient
    // (adjoint) or FP32 staging buffers
    const size_t N = (size_t)src->n;
    CF_TRY(dalloc(c, &c->d_diag32, N));
    CF_TRY(dalloc(c, &c->d_rD32, N));
    CF_TRY(dalloc(c, &c->d_psi, N));
    CF_TRY(dalloc(c, &c->d_b, N));
    CF_TRY(dalloc(c, &c->d_r64, N));
    CF_TRY(dalloc(c, &c->d_io64, N));
    CF_TRY(dalloc(c, &c->d_io64b, N));
    CF_TRY(dalloc(c, &c->d_r0, N));
    CF_TRY(dalloc(c, &c->d_rA, N));
    CF_TRY(dalloc(c, &c->d_W0, N));
    CF_TRY(dalloc(c, &c->d_W1, N));
    CF_TRY(dalloc(c, &c->d_Z0, N));
    CF_TRY(dalloc(c, &c->d_Z1, N));
    CF_TRY(dalloc(c, &c->d_P, 2 * N));
    CF_TRY(dalloc(c, &c->d_Q, 2 * N));
    CF_TRY(dalloc(c, &c->d_T, N));
    CF_TRY(dalloc(c, &c->d_D, 3 * N));
    CF_CUDA(cudaMemsetAsync(c->d_D, 0, sizeof(float) * 3 * N, c->stream));
    CF_CUDA(cudaMemsetAsync(c->d_r64, 0, sizeof(double) * N, c->stream));
    CF_CUDA(cudaStreamSynchronize(c->stream));
    c->hasTopo = true;
    c->hasCoeffs = true;
    CF_TRY(context_clone_sync(src, c));
    guard.c = nullptr;
    *out = c;
    return CF_OK;
}

int context_clone_sync(cf_context* src, cf_context* c)
{
    // the matrix: src's arrays, read only (they stay in src's allocations)
    c->d_sliceOff = src->d_sliceOff;
    c->d_col = src->d_col;
    c->d_col16 = src->d_col16;
    c->d_pcol16 = src->d_pcol16;
    c->d_eface = src->d_eface;
    c->d_perm = src->d_perm;
    c->d_low = src->d_low;
    c->d_upp = src->d_upp;
    c->d_val32 = src->d_val32;
    c->d_pval32 = src->d_pval32;
    c->d_val64 = src->d_val64;
    c->d_valT64 = src->d_valT64;
    c->d_diagIn = src->d_diagIn;
    c->d_upper = src->d_upper;
    c->d_lower = src->d_lower;
    c->d_diag64 = src->d_diag64;
    c->d_u = src->d_u;
    c->lduReady = src->lduReady;
    c->d_own = src->d_own;
    c->d_losS = src->d_losS;
    c->d_los = src->d_los;
    c->d_uppI = src->d_uppI;
    c->d_lowI = src->d_lowI;
    c->d_face32 = src->d_face32;
    c->hasLower = src->hasLower;
    c->val32Sym = src->val32Sym;
    c->transposed = src->transposed;
    c->waitPolls = src->waitPolls;
    cf_spmv_config k;
    CF_TRY(cf_get_spmv_config(src, &k));
    return cf_set_spmv_config(c, &k);
}

}  // namespace cf

extern "C" int cf_set_coeffs(cf_context* c, const double* diag, const double* upper,
                             const double* lower, double* tConvert)
{
    if (!c) return fail(CF_ERR_INVALID_ARG, "context is NULL");
    if (!c->hasTopo) return fail(CF_ERR_NO_TOPOLOGY, "cf_set_topology has not been called");
    if (!diag || (c->nf > 0 && !upper)) return fail(CF_ERR_INVALID_ARG, "NULL coefficient array");
    CF_CUDA(cudaSetDevice(c->device));
    const double t0 = wall_now();
    CF_CUDA(cudaMemcpyAsync(c->d_diagIn, diag, sizeof(double) * c->n, cudaMemcpyHostToDevice,
                            c->stream));
    if (c->nf > 0)
    {
        CF_CUDA(cudaMemcpyAsync(c->d_upper, upper, sizeof(double) * c->nf, cudaMemcpyHostToDevice,
                                c->stream));
        if (lower)
            CF_CUDA(cudaMemcpyAsync(c->d_lower, lower, sizeof(double) * c->nf,
                                    cudaMemcpyHostToDevice, c->stream));
    }
    c->hasLower = lower != nullptr;
    CF_TRY(stage_coeffs_from_device(c));
    CF_CUDA(cudaStreamSynchronize(c->stream));
    if (tConvert) *tConvert = wall_now() - t0;
    return CF_OK;
}

extern "C" int cf_set_coeffs_device(cf_context* c, const double* diag, const double* upper,
                                    const double* lower)
{
    if (!c) return fail(CF_ERR_INVALID_ARG, "context is NULL");
    if (!c->hasTopo) return fail(CF_ERR_NO_TOPOLOGY, "cf_set_topology has not been called");
    if (!diag || (c->nf > 0 && !upper)) return fail(CF_ERR_INVALID_ARG, "NULL coefficient array");
    CF_CUDA(cudaSetDevice(c->device));
    CF_CUDA(cudaMemcpyAsync(c->d_diagIn, diag, sizeof(double) * c->n, cudaMemcpyDeviceToDevice,
                            c->stream));
    if (c->nf > 0)
    {
        CF_CUDA(cudaMemcpyAsync(c->d_upper, upper, sizeof(double) * c->nf,
                                cudaMemcpyDeviceToDevice, c->stream));
        if (lower)
            CF_CUDA(cudaMemcpyAsync(c->d_lower, lower, sizeof(double) * c->nf,
                                    cudaMemcpyDeviceToDevice, c->stream));
    }
    c->hasLower = lower != nullptr;
    return stage_coeffs_from_device(c);
}
