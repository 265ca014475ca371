// cf_static.cu -- an LDU SpMV with fused dot product that allocates nothing.
//
// Who needs it: code that runs where device allocation is not allowed --
// inside a region being captured into a CUDA graph by someone else, on a
// solver thread that must not take the allocator's locks, or in host
// frameworks that hand out only their own pre-allocated device buffers.
// Such callers cannot use a cf_context (its set-up allocates) nor anything
// that calls cudaMalloc behind their back.
//
// The kernel is the row-per-thread LDU product of the reference's
// ldu_spmv_dotw, one thread per cell and one FP64 partial of w.y per block
// of 256 threads.  The partials need scratch memory: here it is a
// file-scope static __device__ array sized for kMaxGroups blocks, so the
// entry point accepts at most kMaxGroups * 256 = 16,777,216 cells.  Every
// GPU that loads this library keeps that array (512 KiB + 256 B) until the
// process exits.
#include "cudafoam.h"

#include <cuda_runtime.h>

#include <mutex>
#include <string>

namespace cf {
int fail(int code, const std::string& msg);
}

namespace {

constexpr int kBlock = 256;
constexpr int kMaxGroups = 65536;                 // partial sums (one per block)
constexpr int kTicketSlot = kMaxGroups;           // completion counter lives here
constexpr int kScratchDoubles = kMaxGroups + 32;  // + one 256-byte line for the counter

// The scratch array.  Host code must not pass this name to a kernel: on the
// host it is only a stand-in for the symbol, not a device address (a kernel
// given it would fault, or on systems where the GPU can reach host memory
// silently use the wrong memory).  The device address comes from
// cudaGetSymbolAddress, once per CUDA context (see scratch_for_current_context).
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

// Device addresses of the array, one per CUDA context that has called.  An
// address from cudaGetSymbolAddress belongs to the context current at the
// lookup, so the key is that context (cuCtxGetCurrent, fetched through the
// runtime's driver entry point so the library does not link libcuda): a
// driver-API caller that makes another context current on the same device
// gets its own lookup.
struct ScratchEntry
{
    void* ctx;
    double* ptr;
};
constexpr int kMaxEntries = 64;
ScratchEntry g_scratch[kMaxEntries];
int g_scratchCount = 0;
std::mutex g_scratchMutex;

typedef int (*CtxGetCurrentFn)(void**);

int current_context(void** out)
{
    static CtxGetCurrentFn fn = nullptr;
    static cudaError_t fnStatus = cudaErrorUnknown;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        fnStatus = cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000,
                                                    cudaEnableDefault, &q);
        if (fnStatus == cudaSuccess && q == cudaDriverEntryPointSuccess && f)
            fn = (CtxGetCurrentFn)f;
        else if (fnStatus == cudaSuccess)
            fnStatus = cudaErrorSymbolNotFound;
    });
    if (!fn)
        return cf::fail(CF_ERR_CUDA, std::string("cuCtxGetCurrent entry point: ") +
                                         cudaGetErrorString(fnStatus));
    *out = nullptr;
    if (fn(out) != 0 || !*out)
        return cf::fail(CF_ERR_CUDA, "cuCtxGetCurrent: no current CUDA context");
    return CF_OK;
}

// The scratch address for the current context.  The lookup itself is not a
// stream operation but may load the module on first use, which a stream
// capture in progress must not see: a first call on a context while `s` is
// capturing is refused with a message saying so.
int scratch_for_current_context(cudaStream_t s, double** out)
{
    // the capture query also initialises the runtime (and the primary
    // context) on a thread whose first CUDA call this is
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    const cudaError_t ce = cudaStreamIsCapturing(s, &cs);
    if (ce != cudaSuccess) cudaGetLastError();
    void* ctx = nullptr;
    int rc = current_context(&ctx);
    if (rc != CF_OK) return rc;
    std::lock_guard<std::mutex> lock(g_scratchMutex);
    for (int i = 0; i < g_scratchCount; ++i)
        if (g_scratch[i].ctx == ctx)
        {
            *out = g_scratch[i].ptr;
            return CF_OK;
        }
    if (ce != cudaSuccess || cs != cudaStreamCaptureStatusNone)
        return cf::fail(CF_ERR_UNSUPPORTED,
                        "cf_ldu_spmv_dot_noalloc: the first call in a CUDA context looks up the "
                        "scratch array's device address and must be made outside stream capture; "
                        "make one call (any size) before capturing");
    if (g_scratchCount == kMaxEntries)
        return cf::fail(CF_ERR_TOO_LARGE, "cf_ldu_spmv_dot_noalloc: more than 64 CUDA contexts");
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
        return cf::fail(CF_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") +
                                         cudaGetErrorString(e));
    g_scratch[g_scratchCount++] = {ctx, (double*)p};
    *out = (double*)p;
    return CF_OK;
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double block_sum(double v, double* sh)
{
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    __syncthreads();
    v = warp_sum(v);
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double t = 0.0;
    if (wid == 0)
    {
        t = lane < kBlock / 32 ? sh[lane] : 0.0;
        t = warp_sum(t);
    }
    return t;  // valid in warp 0
}

// y = A x (diag, then owner-side faces in ownerStart order, then
// neighbour-side faces in losort order; separately rounded products and
// sums) and dot = sum w.y: one partial per block in scratch, the last block
// to finish folds them in block order.
__global__ void __launch_bounds__(kBlock)
    k_ldu_spmv_dot_noalloc(int n, const float* __restrict__ diag, const float* __restrict__ upper,
                           const float* __restrict__ lower, const int* __restrict__ low,
                           const int* __restrict__ upp, const int* __restrict__ ownStart,
                           const int* __restrict__ losort, const int* __restrict__ losortStart,
                           const float* __restrict__ x, const float* __restrict__ w,
                           float* __restrict__ y, double* dot, double* scratch)
{
    __shared__ double sh[kBlock / 32];
    __shared__ bool amLast;
    const int i = blockIdx.x * kBlock + threadIdx.x;
    double acc = 0.0;
    if (i < n)
    {
        float sum = __fmul_rn(diag[i], x[i]);
        for (int f = ownStart[i]; f < ownStart[i + 1]; ++f)
            sum = __fadd_rn(sum, __fmul_rn(upper[f], x[upp[f]]));
        for (int k = losortStart[i]; k < losortStart[i + 1]; ++k)
        {
            const int f = losort[k];
            sum = __fadd_rn(sum, __fmul_rn(lower[f], x[low[f]]));
        }
        y[i] = sum;
        if (w) acc = (double)w[i] * (double)sum;
    }
    if (!dot) return;
    const double part = block_sum(acc, sh);
    unsigned int* ticket = reinterpret_cast<unsigned int*>(scratch + kTicketSlot);
    if (threadIdx.x == 0)
    {
        scratch[blockIdx.x] = part;
        __threadfence();
        amLast = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!amLast) return;
    __threadfence();
    double t = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += kBlock) t += __ldcg(scratch + b);
    t = block_sum(t, sh);
    if (threadIdx.x == 0)
    {
        *dot = t;
        *ticket = 0u;
    }
}

}  // namespace

extern "C" int cf_ldu_spmv_dot_noalloc(int32_t nCells, const float* diag, const float* upper,
                                       const float* lower, const int32_t* lowAddr,
                                       const int32_t* uppAddr, const int32_t* ownStartAddr,
                                       const int32_t* losortAddr,
                                       const int32_t* losortStartAddr, const float* x,
                                       const float* w, float* y, double* dot, void* stream)
{
    if (nCells <= 0) return cf::fail(CF_ERR_INVALID_ARG, "nCells must be > 0");
    const long long groups = ((long long)nCells + kBlock - 1) / kBlock;
    if (groups > kMaxGroups)
        return cf::fail(CF_ERR_TOO_LARGE,
                        "cf_ldu_spmv_dot_noalloc: nCells " + std::to_string(nCells) +
                            " exceeds the fixed scratch limit of " +
                            std::to_string((long long)kMaxGroups * kBlock) + " cells");
    // every addressing array is read for any row that has faces, so none
    // may be NULL (a mesh without faces passes any valid device pointer)
    if (!diag || !upper || !lowAddr || !uppAddr || !ownStartAddr || !losortAddr ||
        !losortStartAddr || !x || !y)
        return cf::fail(CF_ERR_INVALID_ARG, "cf_ldu_spmv_dot_noalloc: NULL device pointer");
    if (!lower) lower = upper;
    cudaStream_t s = (cudaStream_t)stream;
    double* scratch = nullptr;
    int rc = scratch_for_current_context(s, &scratch);
    if (rc != CF_OK) return rc;
    if (dot)
    {
        // the counter must start at zero; the array keeps the last call's
        // contents otherwise
        cudaError_t e = cudaMemsetAsync(scratch + kTicketSlot, 0, sizeof(unsigned int), s);
        if (e != cudaSuccess)
            return cf::fail(CF_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
    }
    k_ldu_spmv_dot_noalloc<<<(unsigned)groups, kBlock, 0, s>>>(
        nCells, diag, upper, lower, lowAddr, uppAddr, ownStartAddr, losortAddr, losortStartAddr, x,
        w, y, dot, scratch);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return cf::fail(CF_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    return CF_OK;
}
