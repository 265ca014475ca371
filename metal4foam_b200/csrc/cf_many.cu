// cf_many.cu -- many independent systems, each in its own context, solved
// concurrently: a pool of host threads, each with its own CUDA stream,
// stages and solves its share one system after another (cf_set_coeffs_device
// + cf_solve_device, unchanged).  Small systems fill few SMs and their
// kernels are short; on separate streams their launches and host
// synchronisations overlap.  Every system gets exactly what cf_solve_device
// on it alone returns (same kernels, same grids, same order of reductions).
#include "cudafoam.h"
#include "cf_host.hpp"

#include <algorithm>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

using namespace cf;

extern "C" int cf_solve_many_device(cf_context* const* ctx, int32_t count, int32_t solver,
                                    double* const* psi, const double* const* source,
                                    const double* const* diag, const double* const* upper,
                                    const double* const* lower, const cf_options* opts,
                                    int32_t streams, cf_performance* perf)
{
    if (count < 0 || !opts || !perf || (count > 0 && (!ctx || !psi || !source)))
        return fail(CF_ERR_INVALID_ARG, "NULL argument or negative count");
    if (streams < 1 || streams > 64) return fail(CF_ERR_INVALID_ARG, "streams must be in [1, 64]");
    for (int i = 0; i < count; ++i)
        if (!ctx[i] || !psi[i] || !source[i] || (diag && (!diag[i] || !upper[i])))
            return fail(CF_ERR_INVALID_ARG, "NULL context or array of system " +
                                                std::to_string(i));
    for (int i = 0; i < count; ++i)
        for (int k = 0; k < i; ++k)
            if (ctx[k] == ctx[i])
                return fail(CF_ERR_INVALID_ARG, "a context appears twice (one system each)");
    // the worker streams are created on one device and only that device is
    // synchronised: every context must live there
    for (int i = 1; i < count; ++i)
        if (ctx[i]->device != ctx[0]->device)
            return fail(CF_ERR_INVALID_ARG, "system " + std::to_string(i) + " is on device " +
                                                std::to_string(ctx[i]->device) + ", system 0 on " +
                                                std::to_string(ctx[0]->device) +
                                                ": all contexts must share one device");
    if (count == 0) return CF_OK;
    // inputs produced by earlier work on any stream are complete
    {
        const cudaError_t e = cudaSetDevice(ctx[0]->device);
        if (e != cudaSuccess) return fail(CF_ERR_CUDA, cudaGetErrorString(e));
        const cudaError_t s = cudaDeviceSynchronize();
        if (s != cudaSuccess) return fail(CF_ERR_CUDA, cudaGetErrorString(s));
    }
    // largest systems first, each to the least-loaded worker
    const int W = std::min<int>(streams, count);
    std::vector<int> order(count);
    std::iota(order.begin(), order.end(), 0);
    auto load = [&](int i) { return (long long)ctx[i]->n + (long long)ctx[i]->nf; };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return load(a) > load(b); });
    std::vector<std::vector<int>> share(W);
    std::vector<long long> work(W, 0);
    for (int i : order)
    {
        const int w = (int)(std::min_element(work.begin(), work.end()) - work.begin());
        share[w].push_back(i);
        work[w] += load(i);
    }
    std::vector<cudaStream_t> st(W, nullptr);
    for (int w = 0; w < W; ++w)
    {
        const cudaError_t e = cudaStreamCreateWithFlags(&st[w], cudaStreamNonBlocking);
        if (e != cudaSuccess)
        {
            for (int k = 0; k < w; ++k) cudaStreamDestroy(st[k]);
            return fail(CF_ERR_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
        }
    }
    std::vector<int> rc(count, CF_OK);
    std::vector<std::string> msg(count);
    auto worker = [&](int w) {
        for (int i : share[w])
        {
            cf_context* c = ctx[i];
            cudaStream_t saved = c->stream;
            c->stream = st[w];
            int r = CF_OK;
            if (diag) r = cf_set_coeffs_device(c, diag[i], upper[i], lower ? lower[i] : nullptr);
            if (r == CF_OK) r = cf_solve_device(c, solver, psi[i], source[i], opts, &perf[i]);
            if (r != CF_OK) msg[i] = cf_last_error();
            c->stream = saved;
            rc[i] = r;
        }
    };
    std::vector<std::thread> pool;
    std::vector<int> inline_shares;   // shares whose thread could not be started
    pool.reserve(W);
    for (int w = 1; w < W; ++w)
    {
        try
        {
            pool.emplace_back(worker, w);
        }
        catch (...)
        {
            inline_shares.push_back(w);   // no exception crosses the C ABI
        }
    }
    worker(0);
    for (int w : inline_shares) worker(w);
    for (auto& t : pool) t.join();
    for (int w = 0; w < W; ++w)
    {
        cudaStreamSynchronize(st[w]);
        cudaStreamDestroy(st[w]);
    }
    for (int i = 0; i < count; ++i)
        if (rc[i] != CF_OK) return fail(rc[i], "system " + std::to_string(i) + ": " + msg[i]);
    return CF_OK;
}
