// simt.hpp -- a small SIMT emulator that lets Metal compute-kernel source
// (the reference's src/metal4Foam/shaders/metalFoamKernels.metal) compile
// and run unchanged as C++ on the CPU (TEST INFRASTRUCTURE ONLY: it builds
// the reference's own kernels into oracle/_ref/ to pin the oracle).
//
// Every thread of a thread group runs as a fiber (ucontext).  Thread groups
// run one after another.  simd_sum() and threadgroup_barrier() park the
// calling fiber until all participants arrive:
//   * simd_sum(v) over the 32 lanes of a simd group, combined as a 5-level
//     xor butterfly (offsets 16, 8, 4, 2, 1) -- every lane gets the same
//     value; Apple does not document its hardware order, this is the order
//     the oracle restates;
//   * threadgroup_barrier(): all threads of the group.
// Metal's address-space qualifiers become empty macros, except that
// `threadgroup` arrays declared inside a kernel are mapped onto one shared
// array per emulator (the kernels' only threadgroup array is `sh`).
#pragma once

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <ucontext.h>

#include <functional>

typedef unsigned int uint;
typedef unsigned short ushort;

namespace simt {

constexpr int kMaxThreads = 1024;
constexpr int kSimd = 32;
constexpr size_t kStack = 64 * 1024;

using Body = std::function<void(uint gid, ushort lane, ushort sgid, ushort nsg, ushort lid,
                                uint tgid)>;

struct Group
{
    int nthreads = 0;
    uint tgid = 0;
    const Body* body = nullptr;
    ucontext_t sched;
    ucontext_t ctx[kMaxThreads];
    char* stacks = nullptr;
    bool done[kMaxThreads];
    int cur = 0;
    // barrier
    int barArrived = 0;
    unsigned barGen = 0;
    // simd_sum
    float simdVal[kMaxThreads / kSimd][kSimd];
    int simdArrived[kMaxThreads / kSimd];
    unsigned simdGen[kMaxThreads / kSimd];
    float simdRes[kMaxThreads / kSimd];
};

inline Group& group()
{
    static Group g;
    return g;
}

inline void park()
{
    Group& g = group();
    swapcontext(&g.ctx[g.cur], &g.sched);
}

inline void trampoline()
{
    Group& g = group();
    const int lid = g.cur;
    const uint gid = g.tgid * (uint)g.nthreads + (uint)lid;
    (*g.body)(gid, (ushort)(lid % kSimd), (ushort)(lid / kSimd), (ushort)(g.nthreads / kSimd),
              (ushort)lid, g.tgid);
    g.done[lid] = true;
    // returning resumes uc_link (the scheduler)
}

inline float butterfly(const float* v)
{
    float a[kSimd], b[kSimd];
    memcpy(a, v, sizeof(a));
    for (int off = kSimd / 2; off >= 1; off >>= 1)
    {
        for (int l = 0; l < kSimd; ++l) b[l] = a[l] + a[l ^ off];
        memcpy(a, b, sizeof(a));
    }
    return a[0];
}

inline float simd_sum_impl(float v)
{
    Group& g = group();
    const int lid = g.cur;
    const int sg = lid / kSimd;
    g.simdVal[sg][lid % kSimd] = v;
    const unsigned gen = g.simdGen[sg];
    if (++g.simdArrived[sg] == kSimd)
    {
        g.simdRes[sg] = butterfly(g.simdVal[sg]);
        g.simdArrived[sg] = 0;
        g.simdGen[sg] = gen + 1;
    }
    else
    {
        while (g.simdGen[sg] == gen) park();
    }
    return g.simdRes[sg];
}

inline void barrier_impl()
{
    Group& g = group();
    const unsigned gen = g.barGen;
    if (++g.barArrived == g.nthreads)
    {
        g.barArrived = 0;
        g.barGen = gen + 1;
    }
    else
    {
        while (g.barGen == gen) park();
    }
}

// Run `groups` thread groups of `tgsize` threads (a multiple of 32).
inline void dispatch(uint groups, int tgsize, const Body& body)
{
    Group& g = group();
    if (!g.stacks) g.stacks = (char*)malloc(kStack * kMaxThreads);
    g.nthreads = tgsize;
    g.body = &body;
    for (uint t = 0; t < groups; ++t)
    {
        g.tgid = t;
        g.barArrived = 0;
        g.barGen = 0;
        memset(g.simdArrived, 0, sizeof(g.simdArrived));
        memset(g.simdGen, 0, sizeof(g.simdGen));
        for (int l = 0; l < tgsize; ++l)
        {
            g.done[l] = false;
            getcontext(&g.ctx[l]);
            g.ctx[l].uc_stack.ss_sp = g.stacks + kStack * (size_t)l;
            g.ctx[l].uc_stack.ss_size = kStack;
            g.ctx[l].uc_link = &g.sched;
            makecontext(&g.ctx[l], (void (*)())trampoline, 0);
        }
        int remaining = tgsize;
        while (remaining > 0)
        {
            for (int l = 0; l < tgsize; ++l)
            {
                if (g.done[l]) continue;
                g.cur = l;
                swapcontext(&g.sched, &g.ctx[l]);
                if (g.done[l]) --remaining;
            }
        }
    }
}

}  // namespace simt

// ---------------------------------------------------------------- Metal names

namespace metal {
enum class mem_flags { mem_none = 0, mem_device = 1, mem_threadgroup = 2 };
inline float simd_sum(float v) { return simt::simd_sum_impl(v); }
inline void threadgroup_barrier(mem_flags) { simt::barrier_impl(); }
}  // namespace metal

// the one threadgroup array of the kernels
extern float simt_tg_sh[32];

#define kernel
#define device
#define constant
#define threadgroup extern
#define sh simt_tg_sh
// tg_sum takes the threadgroup array as a parameter; with the array global
// the parameter is dropped (definition and calls alike)
#define tg_sum(v_, sh_, lane_, sgid_, nsg_) simt_tg_sum(v_, lane_, sgid_, nsg_)
