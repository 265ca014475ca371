"""SpMV launch shapes and the autotuner: every shape (SELL-32 or the
reference's ownerStart/losort addressing read directly; row per thread up
to warp per row; 128/256/512-thread blocks) forms A x bit-identically to
the default shape, solves in any shape converge like the default one, and
the autotuner times all shapes and returns one of them."""
import numpy as np
import pytest

from metal4foam_b200 import _lib, mesh

pytestmark = pytest.mark.gpu

SHAPES = ([("sell32", 32, bs, bits) for bits in (16, 32) for bs in (128, 256, 512)] +
          [("ldu", rpw, bs, 32) for rpw in (32, 8, 4, 1) for bs in (128, 256, 512)])


def make_ctx(s, reorder="auto"):
    ctx = _lib.Context(0, reorder)
    a = s.addr
    ctx.set_topology(a.n, a.nf, *a.arrays())
    ctx.set_coeffs(s.diag, s.upper, s.lower)
    return ctx


@pytest.mark.parametrize("kind", ["sym_permuted", "asym", "sym_identity"])
def test_spmv_bitwise_across_shapes(require_gpu, oracle, kind):
    if kind == "sym_permuted":
        s, reorder = mesh.varcoeff3d((17, 15, 13), seed=21, permute=True), "auto"
    elif kind == "asym":
        s, reorder = mesh.upwind3d((16, 14, 12), seed=22), "auto"
    else:
        s, reorder = mesh.varcoeff3d((40, 33), seed=23, permute=False), "none"
    ctx = make_ctx(s, reorder)
    rng = np.random.default_rng(3)
    x = rng.standard_normal(s.n).astype(np.float32)
    w = rng.standard_normal(s.n).astype(np.float32)
    y0, d0 = ctx.spmv32(x, w)
    yr, _ = oracle.Ldu32View(s).spmv(x, w)
    assert np.array_equal(y0, yr)           # the reference kernel's arithmetic
    for layout, rpw, bs, bits in SHAPES:
        ctx.set_spmv_config(layout=layout, rowsPerWarp=rpw, blockSize=bs, indexBits=bits)
        y, d = ctx.spmv32(x, w)
        assert np.array_equal(y, y0), (layout, rpw, bs, bits)
        assert d == pytest.approx(d0, rel=1e-12, abs=1e-12)
    ctx.close()


def test_cheb_apply_bitwise_across_shapes(require_gpu):
    s = mesh.varcoeff3d((20, 18, 16), seed=24, permute=True)
    ctx = make_ctx(s)
    r = np.random.default_rng(4).standard_normal(s.n).astype(np.float32)
    z0 = ctx.cheb_apply(r, 6, 2.0)
    for layout, rpw, bs, bits in SHAPES:
        ctx.set_spmv_config(layout=layout, rowsPerWarp=rpw, blockSize=bs, indexBits=bits)
        assert np.array_equal(ctx.cheb_apply(r, 6, 2.0), z0), (layout, rpw, bs, bits)
    ctx.close()


@pytest.mark.parametrize("shape", [("sell32", 32, 512), ("ldu", 32, 256), ("ldu", 8, 128),
                                   ("ldu", 1, 256)])
def test_pcg_solve_in_shape(require_gpu, oracle, shape):
    s = mesh.varcoeff3d((24, 22, 20), seed=25, permute=True)
    opts = _lib.default_options(tolerance=1e-8)
    ctx = make_ctx(s)
    x0 = np.zeros(s.n)
    p0 = ctx.solve(_lib.CF_SOLVER_PCG, x0, s.source, opts)
    layout, rpw, bs = shape
    ctx.set_spmv_config(layout=layout, rowsPerWarp=rpw, blockSize=bs)
    xr, _ = oracle.cg64(s)
    for graph in (1, 0):
        x = np.zeros(s.n)
        p = ctx.solve(_lib.CF_SOLVER_PCG, x, s.source, _lib.default_options(tolerance=1e-8,
                                                                            graph=graph))
        assert p.converged and p.finalResidual < 1e-8
        assert abs(p.nIterations - p0.nIterations) <= max(2, 0.02 * p0.nIterations)
        err = np.max(np.abs(x - xr)) / np.max(np.abs(xr))
        err0 = np.max(np.abs(x0 - xr)) / np.max(np.abs(xr))
        assert err < max(10 * err0, 1e-6)
    ctx.close()


@pytest.mark.parametrize("shape", [("sell32", 32, 128), ("ldu", 32, 512), ("ldu", 4, 256)])
def test_bicgstab_solve_in_shape(require_gpu, shape):
    s = mesh.upwind3d((20, 18, 16), seed=26)
    opts = _lib.default_options(tolerance=1e-8, maxIter=3000)
    ctx = make_ctx(s)
    p0 = ctx.solve(_lib.CF_SOLVER_PBICGSTAB, np.zeros(s.n), s.source, opts)
    layout, rpw, bs = shape
    ctx.set_spmv_config(layout=layout, rowsPerWarp=rpw, blockSize=bs)
    x = np.zeros(s.n)
    p = ctx.solve(_lib.CF_SOLVER_PBICGSTAB, x, s.source, opts)
    assert p.converged and p.finalResidual < 1e-8
    assert abs(p.nIterations - p0.nIterations) <= max(3, 0.1 * p0.nIterations)
    r = s.source - mesh.amul_numpy(s, x)
    assert np.sum(np.abs(r)) / p.normFactor == pytest.approx(p.finalResidual, rel=1e-9)
    ctx.close()


def test_transpose_in_ldu_shape(require_gpu):
    """The LDU layout restages its FP32 face coefficients with A^T."""
    s = mesh.upwind3d((12, 11, 10), seed=27)
    ctx = make_ctx(s)
    x = np.random.default_rng(5).standard_normal(s.n).astype(np.float32)
    ctx.set_transpose(True)
    yt0, _ = ctx.spmv32(x, None)
    ctx.set_spmv_config(layout="ldu", rowsPerWarp=8, blockSize=256)
    yt, _ = ctx.spmv32(x, None)
    assert np.array_equal(yt, yt0)
    ctx.set_transpose(False)
    y, _ = ctx.spmv32(x, None)
    ctx.set_spmv_config(layout="sell32", rowsPerWarp=32, blockSize=256)
    y0, _ = ctx.spmv32(x, None)
    assert np.array_equal(y, y0) and not np.array_equal(y, yt)
    ctx.close()


def test_autotune_picks_a_timed_shape(require_gpu):
    s = mesh.varcoeff3d((48, 48, 48), seed=28, permute=True)
    ctx = make_ctx(s)
    best, table = ctx.autotune(reps=10, apply=True)
    assert len(table) == len(SHAPES)
    assert all(ms > 0 for _, ms in table)
    fastest = min(table, key=lambda t: t[1])[0]
    b = best.as_dict()
    keys = ("layout", "rowsPerWarp", "blockSize", "indexBits")
    assert {k: b[k] for k in keys} == {k: fastest[k] for k in keys}
    assert b["rhsTile"] == 0   # the concurrent multi-RHS form is kept
    assert ctx.spmv_config().as_dict() == b
    x = np.zeros(s.n)
    p = ctx.solve(_lib.CF_SOLVER_PCG, x, s.source, _lib.default_options())
    assert p.converged
    ctx.close()


def test_autotune_fused_rhs_tile(require_gpu):
    """With the fused multi-RHS form selected, cf_autotune times the tile."""
    s = mesh.varcoeff3d((32, 32, 32), seed=28, permute=True)
    ctx = make_ctx(s)
    ctx.set_spmv_config(rhsTile=4)
    best, _ = ctx.autotune(reps=5, apply=True)
    assert 1 <= best.as_dict()["rhsTile"] <= 4
    ctx.close()


def test_multi_rhs_tiles_bitwise(require_gpu):
    s = mesh.upwind3d((14, 13, 12), seed=29)
    ctx = make_ctx(s)
    b = np.ascontiguousarray(np.random.default_rng(6).standard_normal((3, s.n)))
    opts = _lib.default_options(tolerance=1e-8)
    ref = np.zeros((3, s.n))
    pr = ctx.solve_multi(_lib.CF_SOLVER_PBICGSTAB, ref, b, opts)
    for tile in (1, 2, 4):
        ctx.set_spmv_config(rhsTile=tile)
        x = np.zeros((3, s.n))
        p = ctx.solve_multi(_lib.CF_SOLVER_PBICGSTAB, x, b, opts)
        assert np.array_equal(x, ref)
        assert [q.nIterations for q in p] == [q.nIterations for q in pr]
    ctx.close()


def test_config_validation_and_topology_change(require_gpu):
    s1 = mesh.varcoeff3d((10, 10, 10), seed=30, permute=True)
    ctx = make_ctx(s1)
    for bad in (dict(layout="sell32", rowsPerWarp=8), dict(blockSize=64), dict(rhsTile=5),
                dict(layout="ldu", rowsPerWarp=16)):
        with pytest.raises(_lib.CudaFoamError) as ei:
            ctx.set_spmv_config(**bad)
        assert ei.value.code == 8
    ctx.set_spmv_config(layout="ldu", rowsPerWarp=4, blockSize=128)
    s2 = mesh.varcoeff3d((20, 10, 5), seed=31, permute=True)
    a = s2.addr
    ctx.set_topology(a.n, a.nf, *a.arrays())
    ctx.set_coeffs(s2.diag, s2.upper, None)
    x = np.random.default_rng(7).standard_normal(s2.n).astype(np.float32)
    y, _ = ctx.spmv32(x, None)
    ctx.set_spmv_config(layout="sell32", rowsPerWarp=32, blockSize=256)
    y0, _ = ctx.spmv32(x, None)
    assert np.array_equal(y, y0)
    ctx.close()


def test_solver_autotune_key_uses_cache(require_gpu, tmp_path, monkeypatch):
    """autotune yes in the cuda sub-dictionary: the first solve on a mesh
    times the shapes and caches the winner; a fresh backend on the same
    mesh applies the cached shape without timing."""
    import json

    from metal4foam_b200 import autotune
    from metal4foam_b200.solver import backend_cache_clear, cudaPCG, lduMatrix
    path = tmp_path / "tune.json"
    monkeypatch.setenv("CUDAFOAM_TUNE_CACHE", str(path))
    s = mesh.varcoeff3d((30, 28, 26), seed=32, permute=True)
    m = lduMatrix(s.addr, s.diag, s.upper)
    ctl = {"solver": "cudaPCG", "tolerance": 1e-7, "cuda": {"autotune": True}}
    psi = np.zeros(s.n)
    p = cudaPCG("p", m, ctl).solve(psi, s.source)
    assert p.converged
    stored = json.loads(path.read_text())
    assert len(stored) == 1
    entry = next(iter(stored.values()))
    backend_cache_clear()
    sol = cudaPCG("p", m, ctl)
    psi2 = np.zeros(s.n)
    p2 = sol.solve(psi2, s.source)
    assert p2.converged
    assert json.loads(path.read_text()) == stored
    assert sol.backend().spmv_config().as_dict() == entry["config"]
    assert autotune.mesh_key(sol.backend().description, s.addr) in stored
    backend_cache_clear()


def test_compact_columns_fall_back_when_offsets_do_not_fit(require_gpu, oracle):
    """A randomly numbered mesh below the RCM threshold keeps columns far
    from their rows: no 16-bit stream is built, indexBits 16 runs the 32-bit
    stream and the autotuner offers only 32-bit SELL shapes."""
    s = mesh.varcoeff3d((40, 40, 40), seed=33, permute=True)      # 64,000 cells
    ctx = make_ctx(s)
    x = np.random.default_rng(8).standard_normal(s.n).astype(np.float32)
    y16, _ = ctx.spmv32(x, None)
    ctx.set_spmv_config(indexBits=32)
    y32, _ = ctx.spmv32(x, None)
    yr, _ = oracle.Ldu32View(s).spmv(x)
    assert np.array_equal(y16, yr) and np.array_equal(y32, yr)
    _, table = ctx.autotune(reps=3, apply=False)
    assert all(t["indexBits"] == 32 for t, _ in table)
    assert len(table) == len(SHAPES) - 3
    ctx.close()


def test_pcg_solve_bitwise_with_either_column_stream(require_gpu):
    """The default shape with 16- or 32-bit columns is the same computation."""
    s = mesh.varcoeff3d((26, 25, 24), seed=34, permute=True)
    ctx = _lib.Context(0, "rcm")
    a = s.addr
    ctx.set_topology(a.n, a.nf, *a.arrays())
    ctx.set_coeffs(s.diag, s.upper, None)
    out = []
    for bits in (16, 32):
        ctx.set_spmv_config(indexBits=bits)
        x = np.zeros(s.n)
        p = ctx.solve(_lib.CF_SOLVER_PCG, x, s.source, _lib.default_options(tolerance=1e-8))
        out.append((x, p.nIterations, p.finalResidual))
    assert np.array_equal(out[0][0], out[1][0]) and out[0][1:] == out[1][1:]
    ctx.close()
