"""The paired copy of the compact column stream is read by kernels compiled
for one slice width each: 4 (2-D quadrilateral meshes), 5 (triangular
prisms: an odd width, whose last entry sits after the pairs) and 6
(hexahedra).  On a mesh of each width the paired kernels must form A x with
the reference kernel's arithmetic (bit for bit against the oracle's
ldu_spmv), apply the Chebyshev polynomial exactly as the 32-bit column
stream does, and give PCG solves identical to the 32-bit stream's; the
BiCGStab kernels of each width must give multi-RHS results equal to single
solves."""
import numpy as np
import pytest

from metal4foam_b200 import _lib, mesh

pytestmark = pytest.mark.gpu

MESHES = {
    4: lambda: mesh.poisson2d(160, 128),
    5: lambda: mesh.prism3d((26, 24, 16), seed=6),
    6: lambda: mesh.varcoeff3d((30, 28, 26), seed=8, permute=True),
}


def make_ctx(s):
    ctx = _lib.Context(0, "rcm")
    a = s.addr
    ctx.set_topology(a.n, a.nf, *a.arrays())
    ctx.set_coeffs(s.diag, s.upper, s.lower)
    return ctx


def asymmetric(s, seed):
    """The same mesh with lower != upper (a convection-like operator)."""
    rng = np.random.default_rng(seed)
    lower = s.upper * (1.0 + 0.4 * rng.uniform(-1.0, 1.0, s.nf))
    diag = 1.05 * (np.bincount(s.addr.lowerAddr, np.abs(s.upper), s.n) +
                   np.bincount(s.addr.upperAddr, np.abs(lower), s.n))
    return mesh.LduSystem(s.name + "_asym", s.addr, diag, s.upper, lower, s.source,
                          np.zeros(s.n), dict(s.meta))


@pytest.mark.parametrize("width", sorted(MESHES))
def test_spmv_and_chebyshev_per_width(require_gpu, oracle, width):
    s = MESHES[width]()
    ctx = make_ctx(s)
    rng = np.random.default_rng(width)
    x = rng.standard_normal(s.n).astype(np.float32)
    w = rng.standard_normal(s.n).astype(np.float32)
    view = oracle.Ldu32View(s)
    y_ref, _ = view.spmv(x, w)
    y16, d16 = ctx.spmv32(x, w)
    assert np.array_equal(y16, y_ref)
    r = rng.standard_normal(s.n).astype(np.float32)
    z16 = ctx.cheb_apply(r, 8, 2.0)
    assert np.array_equal(z16, view.cheb_apply(r, 8, 2.0))
    ctx.set_spmv_config(indexBits=32)
    y32, d32 = ctx.spmv32(x, w)
    assert np.array_equal(y32, y16)
    assert d32 == pytest.approx(d16, rel=1e-12, abs=1e-12)
    assert np.array_equal(ctx.cheb_apply(r, 8, 2.0), z16)
    ctx.close()


@pytest.mark.parametrize("width", sorted(MESHES))
def test_pcg_identical_with_either_stream(require_gpu, oracle, width):
    s = MESHES[width]()
    ctx = make_ctx(s)
    # clusterMaxCells < 0: the graph-driven kernels, not the one-cluster solve
    opts = _lib.default_options(tolerance=1e-8, clusterMaxCells=-1)
    out = []
    for bits in (16, 32):
        ctx.set_spmv_config(indexBits=bits)
        x = np.zeros(s.n)
        p = ctx.solve(_lib.CF_SOLVER_PCG, x, s.source, opts)
        out.append((x, p.nIterations, p.finalResidual))
    assert np.array_equal(out[0][0], out[1][0]) and out[0][1:] == out[1][1:]
    x = out[0][0]
    assert out[0][2] < 1e-8
    r = s.source - oracle.amul(s, x)
    assert np.abs(r).sum() / np.abs(s.source).sum() < 1e-6
    ctx.close()


@pytest.mark.parametrize("width", sorted(MESHES))
def test_bicgstab_multi_rhs_per_width(require_gpu, oracle, width):
    s = asymmetric(MESHES[width](), 40 + width)
    ctx = make_ctx(s)
    opts = _lib.default_options(tolerance=1e-8, maxIter=3000)
    rng = np.random.default_rng(50 + width)
    b = np.ascontiguousarray(np.stack([s.source, rng.standard_normal(s.n),
                                       rng.standard_normal(s.n)]))
    for tile in (0, 4):
        ctx.set_spmv_config(rhsTile=tile)
        psi = np.zeros_like(b)
        perfs = ctx.solve_multi(_lib.CF_SOLVER_PBICGSTAB, psi, b, opts)
        for k in range(3):
            x1 = np.zeros(s.n)
            p1 = ctx.solve(_lib.CF_SOLVER_PBICGSTAB, x1, b[k], opts)
            assert np.array_equal(psi[k], x1), (tile, k)
            assert perfs[k].nIterations == p1.nIterations
            assert perfs[k].converged
            r = b[k] - oracle.amul(s, psi[k])
            assert np.abs(r).sum() / perfs[k].normFactor == pytest.approx(
                perfs[k].finalResidual, rel=1e-9, abs=1e-14)
    ctx.close()
