"""cudaPCG with the aggregation multigrid preconditioner (opt-in,
preconditioner GAMG): the FP64 driver is the reference's, so a converged
solve must meet the same FP64 criterion (sum|b - A psi| / normFactor below
the tolerance, checked here in numpy) and agree with the reference
Chebyshev-Jacobi solve of the same system to the accuracy the tolerance
implies; the hierarchy shrinks to at most nCellsInCoarsestLevel cells;
graph-driven and host-synchronised loops give the same bits."""
import numpy as np
import pytest

from metal4foam_b200 import _lib, mesh

pytestmark = pytest.mark.gpu

PCG = _lib.CF_SOLVER_PCG


def make_ctx(s):
    ctx = _lib.Context(0)
    a = s.addr
    ctx.set_topology(a.n, a.nf, *a.arrays())
    ctx.set_coeffs(s.diag, s.upper, None)
    return ctx


def fp64_residual(s, x, p):
    r = s.source - mesh.amul_numpy(s, x)
    return np.sum(np.abs(r)) / p.normFactor


CASES = [
    ("varcoeff_40_permuted", lambda: mesh.varcoeff3d((40, 40, 40), seed=3, permute=True), {}),
    ("varcoeff_48x40x36", lambda: mesh.varcoeff3d((48, 40, 36), seed=4, permute=False), {}),
    ("poisson2d_128", lambda: mesh.poisson2d(128, 128, seed=5), {}),
    ("varcoeff_30_no_deflation", lambda: mesh.varcoeff3d((30, 28, 26), seed=6, permute=True),
     {"deflate": "off"}),
    ("varcoeff_36_degree3", lambda: mesh.varcoeff3d((36, 34, 32), seed=7, permute=True),
     {"nSweeps": 3, "nCellsInCoarsestLevel": 40, "scaleCorrection": 1.6}),
]


@pytest.mark.parametrize("name,make,kw", CASES, ids=[c[0] for c in CASES])
def test_gamg_converges(require_gpu, name, make, kw):
    s = make()
    ctx = make_ctx(s)
    tol = 1e-7
    xg = np.zeros(s.n)
    pg = ctx.solve(PCG, xg, s.source,
                   _lib.default_options(tolerance=tol, maxIter=5000, preconditioner="GAMG", **kw))
    levels = ctx.gamg_levels()
    xc = np.zeros(s.n)
    pc = ctx.solve(PCG, xc, s.source, _lib.default_options(tolerance=tol, maxIter=5000,
                                                           **{k: v for k, v in kw.items()
                                                              if k == "deflate"}))
    ctx.close()
    assert pg.converged and pg.finalResidual < tol, (name, pg.finalResidual)
    res = fp64_residual(s, xg, pg)
    assert res == pytest.approx(pg.finalResidual, rel=1e-6, abs=1e-15)
    assert res < tol
    # the same system solved both ways: the solutions agree to the accuracy
    # the residual tolerance implies
    scale = np.max(np.abs(xc)) + 1e-30
    assert np.max(np.abs(xg - xc)) / scale < 1e-3, name
    assert pg.nIterations < 5000 and pc.converged
    cap = kw.get("nCellsInCoarsestLevel", 128)
    assert levels[0] == s.n and len(levels) >= 2 and levels[-1] <= cap
    assert all(b < a for a, b in zip(levels, levels[1:])), levels


@pytest.mark.parametrize("dims", [(6, 5), (9, 8, 7)])
def test_gamg_small_meshes(require_gpu, dims):
    """Meshes at or below nCellsInCoarsestLevel still get one coarse level."""
    s = mesh.varcoeff3d(dims, seed=15, permute=False)
    ctx = make_ctx(s)
    x = np.zeros(s.n)
    p = ctx.solve(PCG, x, s.source, _lib.default_options(tolerance=1e-9, preconditioner="GAMG"))
    levels = ctx.gamg_levels()
    ctx.close()
    assert p.converged and fp64_residual(s, x, p) < 1e-9
    assert levels[0] == s.n and len(levels) == 2 and levels[1] < s.n


def test_gamg_graph_and_host_sync_bitwise(require_gpu):
    s = mesh.varcoeff3d((32, 30, 28), seed=8, permute=True)
    ctx = make_ctx(s)
    out = []
    for graph in (1, 0, 1):
        x = np.zeros(s.n)
        p = ctx.solve(PCG, x, s.source, _lib.default_options(tolerance=1e-8, graph=graph,
                                                             preconditioner="GAMG"))
        out.append((x, p.nIterations, p.finalResidual, p.nRestarts))
    ctx.close()
    for x, *rest in out[1:]:
        assert np.array_equal(x, out[0][0]) and rest == list(out[0][1:])


def test_gamg_follows_topology_and_coefficient_changes(require_gpu):
    """A new mesh with the same cell count rebuilds the hierarchy (the same
    result as a fresh context); new coefficients on the same mesh keep the
    hierarchy, whose aggregation followed the first coefficients, and
    re-sum its operators (a correct, converged solve)."""
    s1 = mesh.varcoeff3d((20, 20, 20), seed=9, permute=True)
    s2 = mesh.varcoeff3d((40, 20, 10), seed=10, permute=True)
    s3 = mesh.varcoeff3d((40, 20, 10), seed=11, permute=True)   # same mesh, other values
    assert s1.n == s2.n
    opts = _lib.default_options(tolerance=1e-8, preconditioner="GAMG")
    ctx = make_ctx(s1)
    x = np.zeros(s1.n)
    assert ctx.solve(PCG, x, s1.source, opts).converged
    l1 = ctx.gamg_levels()
    for s in (s2, s3):
        a = s.addr
        ctx.set_topology(a.n, a.nf, *a.arrays())
        ctx.set_coeffs(s.diag, s.upper, None)
        x = np.zeros(s.n)
        p = ctx.solve(PCG, x, s.source, opts)
        assert p.converged and fp64_residual(s, x, p) < 1e-8
        if s is s2:
            ref = make_ctx(s)
            xr = np.zeros(s.n)
            pr = ref.solve(PCG, xr, s.source, opts)
            ref.close()
            assert np.array_equal(x, xr) and p.nIterations == pr.nIterations
    assert ctx.gamg_levels() != l1 or s2.nf != s1.nf
    ctx.close()


def test_gamg_rejects(require_gpu):
    s = mesh.upwind3d((10, 9, 8), seed=12)
    ctx = _lib.Context(0)
    a = s.addr
    ctx.set_topology(a.n, a.nf, *a.arrays())
    ctx.set_coeffs(s.diag, s.upper, s.lower)
    with pytest.raises(_lib.CudaFoamError) as ei:
        ctx.solve(_lib.CF_SOLVER_PBICGSTAB, np.zeros(s.n), s.source,
                  _lib.default_options(preconditioner="GAMG"))
    assert ei.value.code == 8
    for bad in (dict(nSweeps=1), dict(nSweeps=9), dict(nCellsInCoarsestLevel=0),
                dict(nCellsInCoarsestLevel=129), dict(preconditioner=7),
                dict(scaleCorrection=0.0), dict(scaleCorrection=2.0),
                dict(smootherRatio=1.0)):
        kw = dict(preconditioner="GAMG")
        kw.update(bad)
        with pytest.raises(_lib.CudaFoamError) as ei:
            ctx.solve(PCG, np.zeros(s.n), s.source, _lib.default_options(**kw))
        assert ei.value.code == 1, bad
    assert ctx.gamg_levels() == []
    # the multi-RHS (BiCGStab) and batched paths do not offer it
    with pytest.raises(_lib.CudaFoamError) as ei:
        ctx.solve_multi(_lib.CF_SOLVER_PBICGSTAB, np.zeros((2, s.n)),
                        np.ascontiguousarray(np.stack([s.source, s.source])),
                        _lib.default_options(preconditioner="GAMG"))
    assert ei.value.code == 8
    ctx.close()
    sym = mesh.varcoeff3d((8, 7, 6), seed=18, permute=False)
    bt = _lib.Batch(0)
    bt.add_system(sym.addr)
    bt.finalize()
    bt.set_coeffs(0, sym.diag, sym.upper)
    with pytest.raises(_lib.CudaFoamError) as ei:
        bt.solve([np.zeros(sym.n)], [sym.source], _lib.default_options(preconditioner="GAMG"))
    assert ei.value.code == 8
    bt.close()


def test_gamg_whatever_the_spmv_shape(require_gpu):
    """The V-cycle runs its own SELL-32 kernels: under a tuned launch shape
    (another block size, the LDU layout) the GAMG solve is the same bits."""
    s = mesh.varcoeff3d((22, 20, 18), seed=17, permute=True)
    opts = _lib.default_options(tolerance=1e-8, preconditioner="GAMG")
    out = []
    for shape in (None, dict(blockSize=512), dict(layout="ldu", rowsPerWarp=8, blockSize=128)):
        ctx = make_ctx(s)
        if shape:
            ctx.set_spmv_config(**shape)
        x = np.zeros(s.n)
        p = ctx.solve(PCG, x, s.source, opts)
        out.append((x, p.nIterations, p.finalResidual))
        ctx.close()
    for x, *rest in out[1:]:
        assert np.array_equal(x, out[0][0]) and rest == list(out[0][1:])


def test_gamg_solver_surface(require_gpu):
    from metal4foam_b200.solver import FatalError, backend_cache_clear, cudaPCG, lduMatrix
    s = mesh.varcoeff3d((24, 22, 20), seed=13, permute=True)
    m = lduMatrix(s.addr, s.diag, s.upper)
    ctl = {"solver": "cudaPCG", "tolerance": 1e-7,
           "cuda": {"preconditioner": "GAMG", "nSweeps": 2, "nCellsInCoarsestLevel": 64}}
    x = np.zeros(s.n)
    p = cudaPCG("p", m, ctl).solve(x, s.source)
    assert p.converged and fp64_residual(s, x, p) < 1e-7
    with pytest.raises(FatalError):
        cudaPCG("p", m, {"solver": "cudaPCG", "cuda": {"preconditioner": "DIC"}}).solve(
            np.zeros(s.n), s.source)
    backend_cache_clear()


def dense_ldu(n, diag, upper, lo, up):
    A = np.diag(np.asarray(diag, np.float64)).copy()
    A[lo, up] += upper
    A[up, lo] += upper
    return A


@pytest.mark.parametrize("deflate", ["off", "on"])
def test_gamg_galerkin_operators(require_gpu, deflate):
    """Every coarse level is P^T A P of the level above (P the piecewise
    constant prolongation of the exported aggregates; A - diag(A 1) on
    level 0 when deflating), its faces in LDU order, every aggregate a
    connected set of cells."""
    s = mesh.varcoeff3d((14, 12, 10), seed=14, permute=True)
    ctx = make_ctx(s)
    x = np.zeros(s.n)
    p = ctx.solve(PCG, x, s.source, _lib.default_options(
        tolerance=1e-8, preconditioner="GAMG", nCellsInCoarsestLevel=8, deflate=deflate))
    assert p.converged
    assert bool(p.deflated) == (deflate == "on")
    levels = ctx.gamg_levels()
    assert len(levels) >= 3 and levels[-1] <= 8
    a = s.addr
    A = dense_ldu(s.n, s.diag, s.upper, a.lowerAddr, a.upperAddr)
    if deflate == "on" and not p.polished:   # a polish restages the exact operator
        A = A - np.diag(A.sum(axis=1))
    lo_f, up_f = np.asarray(a.lowerAddr), np.asarray(a.upperAddr)
    for lvl in range(1, len(levels)):
        agg, diag, upper, lo, up = ctx.gamg_export(lvl)
        nfine, ncoarse = levels[lvl - 1], levels[lvl]
        assert agg.shape == (nfine,) and agg.min() == 0 and agg.max() == ncoarse - 1
        assert np.all(np.bincount(agg, minlength=ncoarse) > 0)
        P = np.zeros((nfine, ncoarse))
        P[np.arange(nfine), agg] = 1.0
        Ac_ref = P.T @ A @ P
        Ac = dense_ldu(ncoarse, diag, upper, lo, up)
        scale = np.max(np.abs(Ac_ref))
        assert np.max(np.abs(Ac - Ac_ref)) <= 1e-12 * scale, lvl
        # faces: owner < neighbour, sorted by owner then neighbour, no duplicates
        assert np.all(lo < up)
        key = lo.astype(np.int64) * ncoarse + up
        assert np.all(np.diff(key) > 0)
        # aggregates are connected through the finer level's faces
        adj = [[] for _ in range(nfine)]
        for f_lo, f_up in zip(lo_f, up_f):
            if agg[f_lo] == agg[f_up]:
                adj[f_lo].append(f_up)
                adj[f_up].append(f_lo)
        seen = np.zeros(nfine, bool)
        comps = 0
        for i in range(nfine):
            if seen[i]:
                continue
            comps += 1
            stack = [i]
            seen[i] = True
            while stack:
                u = stack.pop()
                for v in adj[u]:
                    if not seen[v]:
                        seen[v] = True
                        stack.append(v)
        assert comps == ncoarse, lvl
        A, lo_f, up_f = Ac, lo, up
    ctx.close()


def test_gamg_with_driver_controls(require_gpu):
    """The V-cycle body under the driver's other controls: convergence
    tests every 4 iterations, an iteration cap that stops the solve early
    (not converged, residual still consistent), and a minimum iteration
    count that forces iterations past convergence."""
    s = mesh.varcoeff3d((30, 28, 26), seed=16, permute=True)
    ctx = make_ctx(s)
    base = dict(tolerance=1e-8, preconditioner="GAMG")
    x = np.zeros(s.n)
    p = ctx.solve(PCG, x, s.source, _lib.default_options(iterationsPerSync=4, **base))
    assert p.converged and fp64_residual(s, x, p) < 1e-8
    x = np.zeros(s.n)
    p = ctx.solve(PCG, x, s.source, _lib.default_options(maxIter=3, **base))
    assert not p.converged and p.nIterations <= 3
    assert fp64_residual(s, x, p) == pytest.approx(p.finalResidual, rel=1e-6)
    x = np.zeros(s.n)
    p1 = ctx.solve(PCG, x, s.source, _lib.default_options(**base))
    x = np.zeros(s.n)
    p2 = ctx.solve(PCG, x, s.source, _lib.default_options(minIter=p1.nIterations + 5,
                                                          maxIter=5000, **base))
    assert p2.converged and p2.nIterations >= p1.nIterations
    ctx.close()
