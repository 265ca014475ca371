"""Generate tests/golden/msl_kernels.npz from the reference's own kernels.

The reference's kernel source (src/metal4Foam/shaders/metalFoamKernels.metal)
is compiled unchanged for the CPU by ``make -C oracle ref`` (SIMT shim in
oracle/msl_shim) into oracle/_ref/libmslref.so.  This script runs every
kernel on seeded inputs -- two LDU systems (an asymmetric upwind 9x8x7 mesh
and a permuted symmetric variable-coefficient 10x9x8 mesh, 2-3 thread groups
each so the partial sums are exercised) -- and stores inputs and outputs as
golden vectors.  tests/test_oracle_golden.py checks the oracle's C
restatement and, transitively, the CUDA kernels against them.

  make -C oracle ref && python tests/golden/make_golden.py
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from metal4foam_b200 import mesh  # noqa: E402

OUT = os.path.join(HERE, "msl_kernels.npz")


def f32(a):
    return np.ascontiguousarray(a, np.float32)


def u32(a):
    return np.ascontiguousarray(a, np.uint32)


def P(a):
    return a.ctypes.data_as(C.c_void_p)


def systems():
    return {"upwind": mesh.upwind3d((9, 8, 7), seed=21),
            "varperm": mesh.varcoeff3d((10, 9, 8), seed=22, permute=True)}


def run(ref, tag, s, rng, out):
    n = s.n
    a = s.addr
    ng = (n + 255) // 256
    diag = f32(s.diag)
    upper = f32(s.upper)
    lower = f32(s.lower_or_upper)
    addr = [u32(x) for x in (a.lowerAddr, a.upperAddr, a.ownerStartAddr, a.losortAddr,
                             a.losortStartAddr)]
    x, w, r, v, rD, z0, p0, wA, dl, rA0, yA, AyA, sA, zA, tA = (
        f32(rng.standard_normal(n)) for _ in range(15))
    s16 = f32(rng.uniform(0.5, 2.0, 16))
    y = np.zeros(n, np.float32)
    part = np.zeros(ng, np.float32)
    ref.ref_ldu_spmv_dotw(n, P(diag), P(upper), P(lower), *map(P, addr), P(x), P(w), P(y), P(part))
    out[f"{tag}/spmv_dotw/y"] = y.copy()
    out[f"{tag}/spmv_dotw/partials"] = part.copy()
    y2 = np.zeros(n, np.float32)
    ref.ref_ldu_spmv(n, P(diag), P(upper), P(lower), *map(P, addr), P(x), P(y2))
    out[f"{tag}/spmv/y"] = y2
    ww = np.zeros(n, np.float32)
    zz = np.zeros(n, np.float32)
    ref.ref_cheb_init(n, P(r), P(rD), P(ww), P(zz), C.c_float(0.7))
    out[f"{tag}/cheb_init/w"] = ww.copy()
    out[f"{tag}/cheb_init/z"] = zz.copy()
    ref.ref_cheb_step(n, P(r), P(v), P(rD), P(ww), P(zz), C.c_float(0.3), C.c_float(1.1))
    out[f"{tag}/cheb_step/w"] = ww.copy()
    out[f"{tag}/cheb_step/z"] = zz.copy()
    e = np.zeros(n, np.float32)
    ref.ref_emul(n, P(rD), P(p0), P(e))
    out[f"{tag}/emul/out"] = e
    wa2 = np.zeros(n, np.float32)
    ref.ref_pcg_precond_dot(n, P(r), P(rD), P(wa2), P(part))
    out[f"{tag}/precond_dot/wA"] = wa2
    out[f"{tag}/precond_dot/partials"] = part.copy()
    pp = p0.copy()
    ref.ref_pcg_update_p(n, P(pp), P(wA), P(s16))
    out[f"{tag}/update_p/p"] = pp
    d2 = dl.copy()
    r2 = r.copy()
    ref.ref_pcg_update_sol_res(n, P(d2), P(r2), P(p0), P(wA), P(s16), P(part))
    out[f"{tag}/update_sol_res/delta"] = d2
    out[f"{tag}/update_sol_res/rA"] = r2
    out[f"{tag}/update_sol_res/partials"] = part.copy()
    ref.ref_dot_partial(n, P(x), P(w), P(part))
    out[f"{tag}/dot_partial/partials"] = part.copy()
    p3 = p0.copy()
    ref.ref_bicg_update_p(n, P(p3), P(r), P(AyA), P(s16))
    out[f"{tag}/bicg_update_p/p"] = p3
    s3 = np.zeros(n, np.float32)
    ref.ref_bicg_s_res(n, P(s3), P(r), P(AyA), P(s16), P(part))
    out[f"{tag}/bicg_s_res/sA"] = s3
    out[f"{tag}/bicg_s_res/partials"] = part.copy()
    d3 = dl.copy()
    ref.ref_bicg_early_update(n, P(d3), P(yA), P(s16))
    out[f"{tag}/bicg_early_update/delta"] = d3
    d4 = dl.copy()
    r4 = r.copy()
    ref.ref_bicg_update_sol_res(n, P(d4), P(yA), P(zA), P(r4), P(sA), P(tA), P(s16), P(part))
    out[f"{tag}/bicg_update_sol_res/delta"] = d4
    out[f"{tag}/bicg_update_sol_res/rA"] = r4
    out[f"{tag}/bicg_update_sol_res/partials"] = part.copy()
    for name, val in dict(x=x, w=w, r=r, v=v, rD=rD, p0=p0, wA=wA, dl=dl, yA=yA, AyA=AyA,
                          sA=sA, zA=zA, tA=tA, s16=s16).items():
        out[f"{tag}/in/{name}"] = val


def run_reduce(ref, rng, out):
    for count in (2, 37, 300):
        P1 = f32(rng.standard_normal(count))
        P2 = f32(rng.standard_normal(count))
        out[f"reduce/{count}/P1"] = P1
        out[f"reduce/{count}/P2"] = P2
        for mode in range(6):
            for first in (0, 1):
                s = f32(rng.uniform(0.5, 2.0, 16))
                out[f"reduce/{count}/{mode}/{first}/s_in"] = s.copy()
                ref.ref_reduce_scalars(P(P1), P(P2), P(s), count, mode, first)
                out[f"reduce/{count}/{mode}/{first}/s_out"] = s.copy()


def main():
    lib = os.path.join(ROOT, "oracle", "_ref", "libmslref.so")
    if not os.path.exists(lib):
        raise SystemExit("build the reference kernels first: make -C oracle ref")
    ref = C.CDLL(lib)
    for nm in dir(ref):
        pass
    out = {}
    rng = np.random.default_rng(2024)
    for tag, s in systems().items():
        run(ref, tag, s, rng, out)
    run_reduce(ref, rng, out)
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT}: {len(out)} arrays")


if __name__ == "__main__":
    main()
