"""Inner PCG inside one thread-block cluster (meshes up to 16,384 cells,
one row per thread): every work vector in distributed shared memory,
hardware cluster barriers between the phases.  Per row the arithmetic is
the graph path's; the dot products fold in their own order, so the
comparison is on convergence, iteration counts and the solution's error
against an FP64 solve.  Meshes without locality (most columns in another
CTA) take the graph path."""
import numpy as np
import pytest

from metal4foam_b200 import _lib, mesh

pytestmark = pytest.mark.gpu


def run(s, cluster, reorder="auto", **kw):
    ctx = _lib.Context(0, reorder)
    a = s.addr
    ctx.set_topology(a.n, a.nf, *a.arrays())
    ctx.set_coeffs(s.diag, s.upper, s.lower)
    x = np.zeros(s.n)
    l0 = ctx.kernel_launches()
    p = ctx.solve(_lib.CF_SOLVER_PCG, x, s.source,
                  _lib.default_options(clusterMaxCells=0 if cluster else -1, **kw))
    launches = ctx.kernel_launches() - l0
    ctx.close()
    return x, p, launches


def _system(n, low, upp, diag, upper, src):
    a = mesh.ldu_addressing(n, np.array(low, np.int32), np.array(upp, np.int32))
    return mesh.LduSystem("edge", a, np.asarray(diag, float), np.asarray(upper, float), None,
                          np.asarray(src, float), np.zeros(n))


# (name, system, options, reorder, cluster path expected)
CASES = [
    ("poisson2d_128", lambda: mesh.poisson2d(128, 128, seed=3),
     dict(chebyshevOrder=4, maxRestarts=4), "auto", True),
    ("poisson2d_64", lambda: mesh.poisson2d(64, 64, seed=2), {}, "auto", True),
    # 1,023 cells: 16 CTAs of 64 rows, two grid lines each -- too many remote
    # columns, so the graph path runs
    ("varcoeff_33x31", lambda: mesh.varcoeff3d((33, 31), seed=5, permute=False), {}, "auto",
     False),
    ("jacobi_2d", lambda: mesh.varcoeff3d((100, 90), seed=6, permute=False),
     dict(chebyshevOrder=1, maxIter=5000), "auto", True),
    ("no_deflation_2d", lambda: mesh.varcoeff3d((70, 60), seed=7, permute=False),
     dict(deflate="off", tolerance=1e-7), "auto", True),
    ("ips3_2d", lambda: mesh.varcoeff3d((80, 50), seed=8, permute=False),
     dict(iterationsPerSync=3), "auto", True),
    ("permuted_3d_falls_back", lambda: mesh.varcoeff3d((24, 24, 24), seed=4, permute=True),
     {}, "auto", False),
    ("permuted_2d_rcm", lambda: mesh.varcoeff3d((90, 80), seed=9, permute=True), {}, "rcm",
     True),
    ("one_cell", lambda: _system(1, [], [], [2.0], [], [4.0]), {}, "auto", None),
]


@pytest.mark.parametrize("name,make,kw,reorder,expect", CASES, ids=[c[0] for c in CASES])
def test_cluster_matches_graph(require_gpu, oracle, name, make, kw, reorder, expect):
    s = make()
    xg, pg, lg = run(s, False, reorder, **kw)
    xc, pc, lc = run(s, True, reorder, **kw)
    if expect is True:
        assert lc < lg, (name, lc, lg)       # one launch per inner solve
    elif expect is False:
        assert lc == lg and pc.nIterations == pg.nIterations and np.array_equal(xc, xg)
    assert pc.converged == pg.converged and pc.deflated == pg.deflated
    assert pc.initialResidual == pg.initialResidual
    assert abs(pc.nIterations - pg.nIterations) <= max(2, 0.05 * pg.nIterations), \
        (name, pc.nIterations, pg.nIterations)
    if pg.converged:
        assert pc.finalResidual < (kw.get("tolerance", 1e-6))
        r = s.source - mesh.amul_numpy(s, xc)
        # (the residual is ~1e-7 of b: another summation order moves it ~1e-9)
        assert np.sum(np.abs(r)) / pc.normFactor == pytest.approx(pc.finalResidual, rel=1e-6)
        xr, _ = oracle.cg64(s)
        scale = max(np.max(np.abs(xr)), 1e-300)
        err_c = np.max(np.abs(xc - xr)) / scale
        err_g = np.max(np.abs(xg - xr)) / scale
        assert err_c <= max(3 * err_g, 1e-6), (name, err_c, err_g)


def test_cluster_not_used_above_16384_cells(require_gpu):
    s = mesh.poisson2d(130, 128, seed=10)          # 16,640 cells
    _, p1, l1 = run(s, True)
    _, p2, l2 = run(s, False)
    assert l1 == l2 and p1.nIterations == p2.nIterations
