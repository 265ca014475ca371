"""Several right-hand sides on one matrix (the momentum components Ux, Uy,
Uz of one fvMatrix): cf_solve_multi must return, per component, exactly
what cf_solve returns for that component alone -- the same psi bit for bit,
the same iteration and restart counts and residuals -- in both of its forms:
rhsTile 0 (components as concurrent single solves sharing the matrix) and
rhsTile 1..4 (fused passes, every SpMV reading the matrix once for all
components of a pass)."""
import numpy as np
import pytest

from metal4foam_b200 import _lib, mesh

pytestmark = pytest.mark.gpu

BICG = _lib.CF_SOLVER_PBICGSTAB


FORMS = [0, 4]   # rhsTile: concurrent single solves, fused passes of 4


def make_ctx(s, tile=0):
    ctx = _lib.Context(0)
    a = s.addr
    ctx.set_topology(a.n, a.nf, *a.arrays())
    ctx.set_coeffs(s.diag, s.upper, s.lower)
    if tile:
        ctx.set_spmv_config(rhsTile=tile)
    return ctx


def single(ctx, psi0, b, opts):
    psi = psi0.copy()
    p = ctx.solve(BICG, psi, b, opts)
    return psi, p


FIELDS = ("initialResidual", "finalResidual", "nIterations", "nRestarts", "converged",
          "singular", "stagnated", "solved", "normFactor", "finalResSum32", "residualL2")


def assert_same(pm, ps, what):
    for f in FIELDS:
        assert getattr(pm, f) == getattr(ps, f), (what, f, getattr(pm, f), getattr(ps, f))


def rhs_set(s, nrhs, seed):
    rng = np.random.default_rng(seed)
    b = rng.standard_normal((nrhs, s.n))
    b[0] = s.source
    return np.ascontiguousarray(b)


@pytest.mark.parametrize("tile", FORMS)
@pytest.mark.parametrize("nrhs", [1, 2, 3, 4, 5, 9])
def test_multi_equals_single_asymmetric(require_gpu, nrhs, tile):
    s = mesh.upwind3d((20, 18, 16), seed=11)
    opts = _lib.default_options(tolerance=1e-8, maxIter=2000)
    ctx = make_ctx(s, tile)
    b = rhs_set(s, nrhs, 5)
    psi = np.zeros((nrhs, s.n))
    perfs = ctx.solve_multi(BICG, psi, b, opts)
    for k in range(nrhs):
        x1, p1 = single(ctx, np.zeros(s.n), b[k], opts)
        assert_same(perfs[k], p1, k)
        assert np.array_equal(psi[k], x1), k
        assert perfs[k].converged
    ctx.close()


@pytest.mark.parametrize("tile", FORMS)
def test_multi_equals_single_symmetric_permuted(require_gpu, tile):
    s = mesh.varcoeff3d((14, 13, 12), seed=12, permute=True)
    opts = _lib.default_options(tolerance=1e-7, maxIter=3000)
    ctx = make_ctx(s, tile)
    b = rhs_set(s, 3, 6)
    psi0 = np.random.default_rng(7).standard_normal((3, s.n))
    psi = psi0.copy()
    perfs = ctx.solve_multi(BICG, psi, b, opts)
    for k in range(3):
        x1, p1 = single(ctx, psi0[k], b[k], opts)
        assert_same(perfs[k], p1, k)
        assert np.array_equal(psi[k], x1), k
    ctx.close()


@pytest.mark.parametrize("tile", FORMS)
def test_multi_uneven_components_graph_and_host_sync(require_gpu, oracle, tile):
    """Components that need very different work: one already solved, one
    easy, one hard; graph and host-synchronised loops agree bit for bit."""
    s = mesh.upwind3d((16, 15, 14), seed=13)
    ctx = make_ctx(s, tile)
    tight = _lib.default_options(tolerance=1e-13, relTol=0.0, maxIter=5000)
    x0 = np.zeros(s.n)
    ctx.solve(BICG, x0, s.source, tight)
    b = np.ascontiguousarray(np.stack([s.source, 1e-3 * s.source, s.source[::-1].copy()]))
    start = np.stack([x0, np.zeros(s.n), np.zeros(s.n)])
    opts_g = _lib.default_options(tolerance=1e-6, maxIter=2000, graph=1)
    opts_h = _lib.default_options(tolerance=1e-6, maxIter=2000, graph=0)
    a = start.copy()
    pa = ctx.solve_multi(BICG, a, b, opts_g)
    h = start.copy()
    ph = ctx.solve_multi(BICG, h, b, opts_h)
    assert pa[0].solved == 0 and pa[0].nIterations == 0
    assert np.array_equal(a[0], x0)
    for k in range(3):
        assert_same(pa[k], ph[k], k)
        assert np.array_equal(a[k], h[k])
        x1, p1 = single(ctx, start[k], b[k], opts_g)
        assert_same(pa[k], p1, k)
        assert np.array_equal(a[k], x1)
    ctx.close()


@pytest.mark.parametrize("tile", FORMS)
def test_multi_max_iter_and_min_iter(require_gpu, tile):
    s = mesh.upwind3d((12, 11, 10), seed=14)
    ctx = make_ctx(s, tile)
    b = rhs_set(s, 3, 8)
    for kw in (dict(maxIter=0), dict(maxIter=7), dict(minIter=40, tolerance=1e-3),
               dict(maxRestarts=0, maxIter=5)):
        opts = _lib.default_options(**kw)
        psi = np.zeros((3, s.n))
        perfs = ctx.solve_multi(BICG, psi, b, opts)
        for k in range(3):
            x1, p1 = single(ctx, np.zeros(s.n), b[k], opts)
            assert_same(perfs[k], p1, (kw, k))
            assert np.array_equal(psi[k], x1), (kw, k)
    ctx.close()


@pytest.mark.parametrize("tile", FORMS)
def test_multi_device_pointers(require_gpu, tile):
    import torch
    s = mesh.upwind3d((18, 17, 9), seed=15)
    ctx = make_ctx(s, tile)
    b = rhs_set(s, 3, 9)
    opts = _lib.default_options(tolerance=1e-8)
    psi_h = np.zeros((3, s.n))
    ph = ctx.solve_multi(BICG, psi_h, b, opts)
    psi_d = torch.zeros((3, s.n), dtype=torch.float64, device="cuda")
    b_d = torch.from_numpy(b).cuda()
    pd = ctx.solve_multi_device(BICG, psi_d, b_d, opts)
    torch.cuda.synchronize()
    assert np.array_equal(psi_d.cpu().numpy(), psi_h)
    for k in range(3):
        assert_same(pd[k], ph[k], k)
    ctx.close()


@pytest.mark.parametrize("tile", FORMS)
def test_multi_topology_change_rebuilds(require_gpu, tile):
    """A new mesh with the same cell count must not reuse buffers or graphs
    that point into the old topology."""
    s1 = mesh.upwind3d((10, 10, 10), seed=16)
    s2 = mesh.upwind3d((20, 10, 5), seed=17)
    assert s1.n == s2.n
    ctx = make_ctx(s1, tile)
    opts = _lib.default_options(tolerance=1e-8)
    b = rhs_set(s1, 2, 10)
    ctx.solve_multi(BICG, np.zeros((2, s1.n)), b, opts)
    a = s2.addr
    ctx.set_topology(a.n, a.nf, *a.arrays())
    ctx.set_coeffs(s2.diag, s2.upper, s2.lower)
    b2 = rhs_set(s2, 2, 11)
    psi = np.zeros((2, s2.n))
    perfs = ctx.solve_multi(BICG, psi, b2, opts)
    for k in range(2):
        assert perfs[k].converged
        r = b2[k] - mesh.amul_numpy(s2, psi[k])
        assert np.sum(np.abs(r)) / perfs[k].normFactor == pytest.approx(perfs[k].finalResidual,
                                                                         rel=1e-9)
    ctx.close()


def test_concurrent_form_follows_coeffs_and_shape(require_gpu):
    """The concurrent form solves on the context's current matrix: new
    coefficients, the LDU layout and a symmetric matrix after an asymmetric
    one all reach every component."""
    s = mesh.upwind3d((15, 14, 13), seed=18)
    ctx = make_ctx(s)
    opts = _lib.default_options(tolerance=1e-8, maxIter=2000)
    b = rhs_set(s, 3, 13)

    def check():
        psi = np.zeros((3, s.n))
        perfs = ctx.solve_multi(BICG, psi, b, opts)
        for k in range(3):
            x1, p1 = single(ctx, np.zeros(s.n), b[k], opts)
            assert_same(perfs[k], p1, k)
            assert np.array_equal(psi[k], x1), k

    check()
    ctx.set_coeffs(1.5 * s.diag, 0.9 * s.upper, 1.1 * s.lower)
    check()
    ctx.set_spmv_config(layout="ldu", rowsPerWarp=8, blockSize=128)
    check()
    ctx.set_spmv_config()
    ctx.set_coeffs(s.diag, s.upper, None)
    check()
    ctx.close()


def test_multi_rejects(require_gpu):
    s = mesh.upwind3d((6, 5, 4))
    ctx = make_ctx(s)
    opts = _lib.default_options()
    psi = np.zeros((2, s.n))
    b = rhs_set(s, 2, 12)
    with pytest.raises(_lib.CudaFoamError) as ei:
        ctx.solve_multi(_lib.CF_SOLVER_PCG, psi, b, opts)
    assert ei.value.code == 8
    with pytest.raises(_lib.CudaFoamError) as ei:
        _lib.check(_lib.load().cf_solve_multi(ctx.h, BICG, 0, _lib.ptr(psi), _lib.ptr(b),
                                              _lib.C.byref(opts), None))
    assert ei.value.code == 1
    ctx.close()


def test_momentum_64cube_three_components(require_gpu):
    """The multi-RHS configuration: one 64^3 upwind momentum matrix with 3
    right-hand sides; each component converges to 1e-6 and equals its
    single solve."""
    s, rhs = mesh.momentum_multi_rhs()
    rhs = np.ascontiguousarray(rhs)
    ctx = make_ctx(s)
    opts = _lib.default_options(tolerance=1e-6, maxIter=1000)
    psi = np.zeros_like(rhs)
    perfs = ctx.solve_multi(BICG, psi, rhs, opts)
    for k in range(3):
        assert perfs[k].converged and perfs[k].finalResidual < 1e-6
        x1, p1 = single(ctx, np.zeros(s.n), rhs[k], opts)
        assert_same(perfs[k], p1, k)
        assert np.array_equal(psi[k], x1)
        r = rhs[k] - mesh.amul_numpy(s, psi[k])
        assert np.sum(np.abs(r)) / perfs[k].normFactor < 1.01e-6
    ctx.close()


def test_solver_surface_segregated(require_gpu):
    """cudaPBiCGStab.solveSegregated: every component equals solve() on it."""
    from metal4foam_b200.solver import (FatalError, backend_cache_clear, cudaPBiCGStab,
                                        cudaPCG, lduMatrix)
    s = mesh.upwind3d((18, 16, 14), seed=40)
    m = lduMatrix(s.addr, s.diag, s.upper, s.lower)
    ctl = {"solver": "cudaPBiCGStab", "tolerance": 1e-8}
    b = rhs_set(s, 3, 41)
    psi = np.zeros((3, s.n))
    perfs = cudaPBiCGStab("U", m, ctl).solveSegregated(psi, b)
    for k in range(3):
        x = np.zeros(s.n)
        p1 = cudaPBiCGStab("U", m, ctl).solve(x, b[k])
        assert np.array_equal(psi[k], x)
        assert perfs[k].nIterations == p1.nIterations and perfs[k].converged
        assert perfs[k].fieldName == f"U.component({k})"
    with pytest.raises(FatalError):
        sym = mesh.varcoeff3d((6, 5, 4), seed=1)
        cudaPCG("p", lduMatrix(sym.addr, sym.diag, sym.upper), {"solver": "cudaPCG"}) \
            .solveSegregated(np.zeros((2, sym.n)), np.zeros((2, sym.n)))
    backend_cache_clear()
