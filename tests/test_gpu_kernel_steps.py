"""Kernel-level parity of the fused inner-iteration kernels.

Each fused CUDA kernel replaces a run of the reference's kernels
(metalFoamKernels.metal:64-276,372-458, dispatched per iteration by
metalFoamBackend.C:608-906).  cf_inner_step runs one fused kernel exactly as
the inner loop launches it, on random vectors and given alpha, beta, omega;
the oracle's KernelSequence runs the reference's unfused kernels on the same
inputs.  Every vector the fused kernel writes must be bit-identical; every
reduction it folds (FP32 products accumulated in FP64) must equal the FP64
sum of the same products to 1e-12 relative -- the fold order differs, the
products do not.  Checked in the default launch shape and in two others
(the LDU addressing read directly, and warp per row), with and without the
RCM relabelling, on a symmetric permuted pressure matrix, an asymmetric
upwind matrix and a ragged 2-D mesh.
"""
import numpy as np
import pytest

from metal4foam_b200 import _lib, mesh

pytestmark = pytest.mark.gpu

SYSTEMS = {
    "varcoeff_perm": lambda: mesh.varcoeff3d((21, 19, 17), seed=41, permute=True),
    "upwind": lambda: mesh.upwind3d((18, 17, 16), seed=42),
    "ragged_2d": lambda: mesh.varcoeff3d((53, 7), seed=43, permute=True),
}
SHAPES = {
    "default": None,
    "ldu_row": dict(layout="ldu", rowsPerWarp=32, blockSize=256),
    "ldu_warp": dict(layout="ldu", rowsPerWarp=1, blockSize=128),
    "sell512": dict(layout="sell32", rowsPerWarp=32, blockSize=512),
}
ALPHA, BETA, OMEGA = 0.3719, 0.8123, 1.1377   # rounded to FP32 by both sides
TOL = dict(rel=1e-12, abs=1e-30)


def setup(name, reorder, shape):
    s = SYSTEMS[name]()
    ctx = _lib.Context(0, reorder=reorder)
    a = s.addr
    ctx.set_topology(a.n, a.nf, *a.arrays())
    ctx.set_coeffs(s.diag, s.upper, s.lower)
    if SHAPES[shape] is not None:
        ctx.set_spmv_config(**SHAPES[shape])
    return s, ctx


def vecs(n, names, seed):
    rng = np.random.default_rng(seed)
    return {k: rng.standard_normal(n).astype(np.float32) for k in names}


def compare(got, want):
    outs, sums = got
    ref_outs, ref_sums = want
    for k, v in ref_outs.items():
        assert np.array_equal(outs[k], v), f"{k}: {np.count_nonzero(outs[k] != v)} entries differ"
    for a, b in zip(sums, ref_sums):
        assert a == pytest.approx(b, **TOL)


@pytest.mark.parametrize("shape", sorted(SHAPES))
@pytest.mark.parametrize("reorder", ["none", "rcm"])
def test_pcg_kernels_match_reference_sequence(require_gpu, oracle, reorder, shape):
    s, ctx = setup("varcoeff_perm", reorder, shape)
    seq = oracle.KernelSequence(s)
    n = s.n
    order, beta_c, ratio = 8, 2.7, 30.0
    v = vecs(n, ["zIn", "wIn", "rA", "wA", "pOld", "delta", "p", "q"], 1)
    for step in (1, 4, order - 1):
        compare(ctx.inner_step("cheb", n, chebOrder=order, chebStep=step, chebBeta=beta_c,
                               chebRatio=ratio, zIn=v["zIn"], wIn=v["wIn"], rA=v["rA"]),
                seq.cheb_step(v["zIn"], v["wIn"], v["rA"], order, step, beta_c, ratio))
    compare(ctx.inner_step("pcg_p_spmv", n, beta=BETA, wA=v["wA"], pOld=v["pOld"]),
            seq.pcg_p_spmv(v["wA"], v["pOld"], BETA))
    # the update with the next Chebyshev start, and with the Jacobi apply + dot
    compare(ctx.inner_step("pcg_update", n, alpha=ALPHA, chebOrder=order, chebBeta=beta_c,
                           chebRatio=ratio, delta=v["delta"], p=v["p"], rA=v["rA"], q=v["q"]),
            seq.pcg_update(v["delta"], v["p"], v["rA"], v["q"], ALPHA, order, beta_c, ratio))
    compare(ctx.inner_step("pcg_update", n, alpha=ALPHA, chebOrder=1, delta=v["delta"],
                           p=v["p"], rA=v["rA"], q=v["q"]),
            seq.pcg_update(v["delta"], v["p"], v["rA"], v["q"], ALPHA, 1))
    ctx.close()


@pytest.mark.parametrize("shape", sorted(SHAPES))
@pytest.mark.parametrize("name", ["upwind", "ragged_2d"])
def test_bicgstab_kernels_match_reference_sequence(require_gpu, oracle, name, shape):
    s, ctx = setup(name, "rcm", shape)
    seq = oracle.KernelSequence(s)
    n = s.n
    v = vecs(n, ["rA", "rA0", "pOld", "AyAOld", "AyA", "delta", "yA", "zA", "sA", "tA"], 2)
    compare(ctx.inner_step("bicg_ab", n, beta=BETA, omega=OMEGA, rA=v["rA"], pOld=v["pOld"],
                           AyAOld=v["AyAOld"], rA0=v["rA0"]),
            seq.bicg_ab(v["rA"], v["pOld"], v["AyAOld"], v["rA0"], BETA, OMEGA))
    compare(ctx.inner_step("bicg_cd", n, alpha=ALPHA, rA=v["rA"], AyA=v["AyA"]),
            seq.bicg_cd(v["rA"], v["AyA"], ALPHA))
    compare(ctx.inner_step("bicg_e", n, alpha=ALPHA, omega=OMEGA, delta=v["delta"],
                           yA=v["yA"], zA=v["zA"], sA=v["sA"], tA=v["tA"], rA0=v["rA0"]),
            seq.bicg_e(v["delta"], v["yA"], v["zA"], v["sA"], v["tA"], v["rA0"], ALPHA, OMEGA))
    ctx.close()


def test_one_iteration_chains_like_the_reference(require_gpu, oracle):
    """A whole BiCGStab iteration chained through the fused kernels, each
    step's outputs fed to the next with the scalars the reference would
    form from the sums: same vectors as the reference's kernels run in
    sequence."""
    s, ctx = setup("upwind", "rcm", "default")
    seq = oracle.KernelSequence(s)
    n = s.n
    v = vecs(n, ["rA", "pOld", "AyAOld", "delta"], 3)
    rA0 = v["rA"].copy()
    beta, omega = 0.55, 0.9
    ab, sums_ab = ctx.inner_step("bicg_ab", n, beta=beta, omega=omega, rA=v["rA"],
                                 pOld=v["pOld"], AyAOld=v["AyAOld"], rA0=rA0)
    ref_ab, _ = seq.bicg_ab(v["rA"], v["pOld"], v["AyAOld"], rA0, beta, omega)
    assert all(np.array_equal(ab[k], ref_ab[k]) for k in ref_ab)
    rA0rA = float(np.dot(rA0.astype(np.float64), v["rA"].astype(np.float64)))
    alpha = float(np.float32(rA0rA / sums_ab[0]))
    cd, sums_cd = ctx.inner_step("bicg_cd", n, alpha=alpha, rA=v["rA"], AyA=ab["AyA"])
    ref_cd, _ = seq.bicg_cd(v["rA"], ref_ab["AyA"], alpha)
    assert all(np.array_equal(cd[k], ref_cd[k]) for k in ref_cd)
    omega2 = float(np.float32(sums_cd[1] / sums_cd[2]))
    e, _ = ctx.inner_step("bicg_e", n, alpha=alpha, omega=omega2, delta=v["delta"],
                          yA=ab["yA"], zA=cd["zA"], sA=cd["sA"], tA=cd["tA"], rA0=rA0)
    ref_e, _ = seq.bicg_e(v["delta"], ref_ab["yA"], ref_cd["zA"], ref_cd["sA"], ref_cd["tA"],
                          rA0, alpha, omega2)
    assert all(np.array_equal(e[k], ref_e[k]) for k in ref_e)
    ctx.close()


def test_inner_step_rejects_bad_arguments(require_gpu):
    s, ctx = setup("ragged_2d", "none", "default")
    n = s.n
    z = np.zeros(n, np.float32)
    with pytest.raises(_lib.CudaFoamError) as ei:
        ctx.inner_step("cheb", n, chebOrder=8, chebStep=8, zIn=z, wIn=z, rA=z)
    assert ei.value.code == 1
    with pytest.raises(_lib.CudaFoamError) as ei:   # a required input missing
        ctx.inner_step("pcg_p_spmv", n, beta=1.0, wA=z)
    assert ei.value.code == 1
    # the context still solves afterwards
    psi = np.zeros(n)
    p = ctx.solve(_lib.CF_SOLVER_PCG, psi, s.source, _lib.default_options())
    assert p.converged
    ctx.close()
