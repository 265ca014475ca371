"""The on-disk cache of tuned SpMV launch shapes (metal4foam_b200.autotune),
driven by a stand-in context on the CPU: the first call times and stores,
later calls apply the stored shape without timing."""
import json

import pytest

from metal4foam_b200 import _lib, autotune, mesh


class FakeContext:
    description = "cudaFoam: test device"
    reorder = "auto"

    def __init__(self):
        self.tuned = 0
        self.applied = []

    def autotune(self, reps=20, apply=True):
        self.tuned += 1
        best = _lib.spmv_config(layout="ldu", rowsPerWarp=8, blockSize=128, rhsTile=3)
        table = [({"layout": "sell32", "rowsPerWarp": 32, "blockSize": 256, "rhsTile": 4}, 0.2),
                 (best.as_dict(), 0.1)]
        return best, table

    def set_spmv_config(self, **kw):
        self.applied.append(kw)


def test_mesh_key_is_structural():
    a = mesh.varcoeff3d((8, 7, 6), seed=1, permute=False).addr
    b = mesh.varcoeff3d((8, 7, 6), seed=2, permute=False).addr   # same structure, other values
    c = mesh.varcoeff3d((8, 7, 6), seed=1, permute=True).addr
    k = autotune.mesh_key("dev", a)
    assert k == autotune.mesh_key("dev", b)
    assert k != autotune.mesh_key("dev", c)
    assert k != autotune.mesh_key("dev2", a)
    assert k != autotune.mesh_key("dev", a, reorder="none")


def test_tune_once_then_cached(tmp_path, monkeypatch):
    path = tmp_path / "tune.json"
    monkeypatch.setenv("CUDAFOAM_TUNE_CACHE", str(path))
    addr = mesh.poisson2d(20, 10).addr
    ctx = FakeContext()
    cfg = autotune.tuned_config(ctx, addr)
    assert ctx.tuned == 1 and ctx.applied == []
    assert cfg == {"layout": "ldu", "rowsPerWarp": 8, "blockSize": 128, "rhsTile": 3,
                   "indexBits": 16}
    stored = json.loads(path.read_text())
    (key, entry), = stored.items()
    assert key == autotune.mesh_key(ctx.description, addr)
    assert entry["config"] == cfg and len(entry["timings_ms"]) == 2
    ctx2 = FakeContext()
    assert autotune.tuned_config(ctx2, addr) == cfg
    assert ctx2.tuned == 0 and ctx2.applied == [cfg]
    ctx3 = FakeContext()
    autotune.tuned_config(ctx3, addr, retune=True)
    assert ctx3.tuned == 1


def test_unreadable_cache_is_ignored(tmp_path):
    path = tmp_path / "bad.json"
    path.write_text("{not json")
    assert autotune.load_cache(str(path)) == {}
    ctx = FakeContext()
    autotune.tuned_config(ctx, mesh.poisson2d(5, 5).addr, path=str(path))
    assert ctx.tuned == 1
    assert len(json.loads(path.read_text())) == 1


def test_solver_accepts_autotune_key():
    from metal4foam_b200.solver import FatalError, cudaPCG, lduMatrix
    s = mesh.poisson2d(4, 4)
    m = lduMatrix(s.addr, s.diag, s.upper)
    sol = cudaPCG("p", m, {"solver": "cudaPCG", "cuda": {"autotune": True}})
    assert sol.subDict_["autotune"] is True
    with pytest.raises(FatalError):
        cudaPCG("p", m, {"solver": "cudaPCG", "cuda": {"autotunes": True}})
