// mslref.cpp -- the reference's own compute kernels
// (src/metal4Foam/shaders/metalFoamKernels.metal, included unchanged from
// where it lies) compiled for the CPU through simt.hpp, each exported as a
// C function that dispatches ceil(n/256) thread groups of 256 threads, the
// reference's launch geometry (dispatchN, metalFoamBackend.C:286-293;
// reduce_scalars: one group of 256, metalFoamBackend.C:415).
// TEST INFRASTRUCTURE ONLY (builds oracle/_ref/libmslref.so).
#include "simt.hpp"

float simt_tg_sh[32];

#include METAL_KERNEL_SOURCE

namespace {
uint groups_of(uint n) { return (n + 255u) / 256u; }
}

extern "C" {

void ref_ldu_spmv_dotw(uint n, const float* diag, const float* upper, const float* lower,
                       const uint* low, const uint* upp, const uint* ownStart, const uint* losort,
                       const uint* losortStart, const float* x, const float* w, float* y,
                       float* partials)
{
    uint nn = n;
    simt::dispatch(groups_of(n), 256, [&](uint gid, ushort lane, ushort sgid, ushort nsg,
                                          ushort lid, uint tgid) {
        ldu_spmv_dotw(diag, upper, lower, low, upp, ownStart, losort, losortStart, x, w, y,
                      partials, nn, gid, lane, sgid, nsg, lid, tgid);
    });
}

void ref_ldu_spmv(uint n, const float* diag, const float* upper, const float* lower,
                  const uint* low, const uint* upp, const uint* ownStart, const uint* losort,
                  const uint* losortStart, const float* x, float* y)
{
    uint nn = n;
    simt::dispatch(groups_of(n), 256, [&](uint gid, ushort, ushort, ushort, ushort, uint) {
        ldu_spmv(diag, upper, lower, low, upp, ownStart, losort, losortStart, x, y, nn, gid);
    });
}

void ref_cheb_init(uint n, const float* r, const float* rD, float* w, float* z, float c1)
{
    uint nn = n;
    float cc = c1;
    simt::dispatch(groups_of(n), 256, [&](uint gid, ushort, ushort, ushort, ushort, uint) {
        cheb_init(r, rD, w, z, cc, nn, gid);
    });
}

void ref_cheb_step(uint n, const float* r, const float* v, const float* rD, float* w, float* z,
                   float c2, float c3)
{
    uint nn = n;
    float a = c2, b = c3;
    simt::dispatch(groups_of(n), 256, [&](uint gid, ushort, ushort, ushort, ushort, uint) {
        cheb_step(r, v, rD, w, z, a, b, nn, gid);
    });
}

void ref_emul(uint n, const float* a, const float* b, float* out)
{
    uint nn = n;
    simt::dispatch(groups_of(n), 256, [&](uint gid, ushort, ushort, ushort, ushort, uint) {
        emul(a, b, out, nn, gid);
    });
}

void ref_pcg_precond_dot(uint n, const float* rA, const float* rD, float* wA, float* partials)
{
    uint nn = n;
    simt::dispatch(groups_of(n), 256, [&](uint gid, ushort lane, ushort sgid, ushort nsg,
                                          ushort lid, uint tgid) {
        pcg_precond_dot(rA, rD, wA, partials, nn, gid, lane, sgid, nsg, lid, tgid);
    });
}

void ref_pcg_update_p(uint n, float* p, const float* wA, const float* s)
{
    uint nn = n;
    simt::dispatch(groups_of(n), 256, [&](uint gid, ushort, ushort, ushort, ushort, uint) {
        pcg_update_p(p, wA, s, nn, gid);
    });
}

void ref_pcg_update_sol_res(uint n, float* delta, float* rA, const float* p, const float* wA,
                            const float* s, float* partials)
{
    uint nn = n;
    simt::dispatch(groups_of(n), 256, [&](uint gid, ushort lane, ushort sgid, ushort nsg,
                                          ushort lid, uint tgid) {
        pcg_update_sol_res(delta, rA, p, wA, s, partials, nn, gid, lane, sgid, nsg, lid, tgid);
    });
}

void ref_dot_partial(uint n, const float* a, const float* b, float* partials)
{
    uint nn = n;
    simt::dispatch(groups_of(n), 256, [&](uint gid, ushort lane, ushort sgid, ushort nsg,
                                          ushort lid, uint tgid) {
        dot_partial(a, b, partials, nn, gid, lane, sgid, nsg, lid, tgid);
    });
}

void ref_reduce_scalars(const float* P1, const float* P2, float* s, uint count, uint mode,
                        uint firstIter)
{
    uint c = count, m = mode, f = firstIter;
    simt::dispatch(1, 256, [&](uint, ushort lane, ushort sgid, ushort nsg, ushort lid,
                               uint tgid) {
        reduce_scalars(P1, P2, s, c, m, f, lane, sgid, nsg, lid, tgid);
    });
}

void ref_bicg_update_p(uint n, float* p, const float* rA, const float* AyA, const float* s)
{
    uint nn = n;
    simt::dispatch(groups_of(n), 256, [&](uint gid, ushort, ushort, ushort, ushort, uint) {
        bicg_update_p(p, rA, AyA, s, nn, gid);
    });
}

void ref_bicg_s_res(uint n, float* sA, const float* rA, const float* AyA, const float* s,
                    float* partials)
{
    uint nn = n;
    simt::dispatch(groups_of(n), 256, [&](uint gid, ushort lane, ushort sgid, ushort nsg,
                                          ushort lid, uint tgid) {
        bicg_s_res(sA, rA, AyA, s, partials, nn, gid, lane, sgid, nsg, lid, tgid);
    });
}

void ref_bicg_early_update(uint n, float* delta, const float* yA, const float* s)
{
    uint nn = n;
    simt::dispatch(groups_of(n), 256, [&](uint gid, ushort, ushort, ushort, ushort, uint) {
        bicg_early_update(delta, yA, s, nn, gid);
    });
}

void ref_bicg_update_sol_res(uint n, float* delta, const float* yA, const float* zA, float* rA,
                             const float* sA, const float* tA, const float* s, float* partials)
{
    uint nn = n;
    simt::dispatch(groups_of(n), 256, [&](uint gid, ushort lane, ushort sgid, ushort nsg,
                                          ushort lid, uint tgid) {
        bicg_update_sol_res(delta, yA, zA, rA, sA, tA, s, partials, nn, gid, lane, sgid, nsg,
                            lid, tgid);
    });
}

}  // extern "C"
