"""Kernel-level parity on the GPU through the C ABI: FP64 Amul, FP32 SpMV and
the fused Chebyshev-Jacobi apply are bit-exact against the oracle (the
reference's kernel arithmetic, metalFoamKernels.metal:64-194, and OpenFOAM's
Amul order); the fused FP64-accumulated dot is within 1e-12 relative."""
import numpy as np
import pytest

from metal4foam_b200 import _lib, mesh

pytestmark = pytest.mark.gpu

SYSTEMS = {
    "poisson2d_64": lambda: mesh.poisson2d(64, 64, seed=3),
    "varcoeff_perm_20": lambda: mesh.varcoeff3d((20, 18, 17), seed=4, permute=True),
    "upwind_16": lambda: mesh.upwind3d((16, 15, 14), seed=5),
    "ragged_2d": lambda: mesh.varcoeff3d((37, 3), seed=6, permute=True),
}


def make_ctx(s, reorder):
    ctx = _lib.Context(0, reorder=reorder)
    a = s.addr
    ctx.set_topology(a.n, a.nf, *a.arrays())
    ctx.set_coeffs(s.diag, s.upper, s.lower)
    return ctx


@pytest.mark.parametrize("reorder", ["none", "rcm"])
@pytest.mark.parametrize("name", sorted(SYSTEMS))
def test_amul64_bit_exact(require_gpu, oracle, name, reorder):
    s = SYSTEMS[name]()
    ctx = make_ctx(s, reorder)
    x = np.random.default_rng(1).standard_normal(s.n)
    assert np.array_equal(ctx.amul(x), oracle.amul(s, x))
    assert np.array_equal(ctx.amul(x, transpose=True), oracle.amul(s, x, transpose=True))
    ctx.close()


@pytest.mark.parametrize("reorder", ["none", "rcm"])
@pytest.mark.parametrize("name", sorted(SYSTEMS))
def test_spmv32_bit_exact(require_gpu, oracle, name, reorder):
    s = SYSTEMS[name]()
    ctx = make_ctx(s, reorder)
    rng = np.random.default_rng(2)
    x = rng.standard_normal(s.n).astype(np.float32)
    w = rng.standard_normal(s.n).astype(np.float32)
    y, dot = ctx.spmv32(x, w)
    view = oracle.Ldu32View(s)
    yo, _ = view.spmv(x)
    assert np.array_equal(y, yo)
    exact = float(np.dot(w.astype(np.float64), yo.astype(np.float64)))
    assert dot == pytest.approx(exact, rel=1e-12, abs=1e-12)
    ctx.close()


@pytest.mark.parametrize("order", [2, 4, 8])
@pytest.mark.parametrize("name", ["poisson2d_64", "varcoeff_perm_20"])
def test_cheb_apply_bit_exact(require_gpu, oracle, name, order):
    s = SYSTEMS[name]()
    ctx = make_ctx(s, "rcm")
    r = np.random.default_rng(3).standard_normal(s.n).astype(np.float32)
    z = ctx.cheb_apply(r, order, 2.5, 30.0)
    zo = oracle.Ldu32View(s).cheb_apply(r, order, 2.5, 30.0)
    assert np.array_equal(z, zo)
    ctx.close()


def test_bad_addressing_rejected(require_gpu):
    s = mesh.poisson2d(8, 8)
    a = s.addr
    ctx = _lib.Context(0)
    low = a.lowerAddr.copy()
    low[3], low[4] = low[4], low[3]
    with pytest.raises(_lib.CudaFoamError) as ei:
        ctx.set_topology(a.n, a.nf, low, a.upperAddr, a.ownerStartAddr, a.losortAddr,
                         a.losortStartAddr)
    assert ei.value.code == 2
    los = a.losortAddr.copy()
    los[[0, 1]] = los[[1, 0]]
    with pytest.raises(_lib.CudaFoamError):
        ctx.set_topology(a.n, a.nf, a.lowerAddr, a.upperAddr, a.ownerStartAddr, los,
                         a.losortStartAddr)
    with pytest.raises(_lib.CudaFoamError) as ei:
        ctx.amul(np.zeros(a.n))
    assert ei.value.code == 3
    ctx.close()


def test_time_kernel_modes(require_gpu):
    """cf_time_kernel: every kernel id returns a positive time and leaves the
    context usable; the in-iteration Chebyshev timing runs full PCG
    iterations (9 launches each)."""
    s = mesh.varcoeff3d((32, 30, 28), seed=11, permute=True)
    ctx = _lib.Context(0)
    a = s.addr
    ctx.set_topology(a.n, a.nf, *a.arrays())
    ctx.set_coeffs(s.diag, s.upper, None)
    # before any solve there is no inner right-hand side to iterate on
    with pytest.raises(_lib.CudaFoamError) as ei:
        ctx.time_kernel("cheb_step_inner", reps=2)
    assert ei.value.code == 1
    x = np.zeros(s.n)
    ctx.solve(_lib.CF_SOLVER_PCG, x, s.source, _lib.default_options(maxIter=3))
    for k in ctx.KERNELS:
        assert ctx.time_kernel(k, reps=4) > 0.0, k
    l0 = ctx.kernel_launches()
    ctx.time_kernel("cheb_step_inner", reps=3)
    assert ctx.kernel_launches() - l0 >= 27
    x = np.zeros(s.n)
    p = ctx.solve(_lib.CF_SOLVER_PCG, x, s.source, _lib.default_options())
    assert p.converged
    ctx.close()
