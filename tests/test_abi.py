"""The C-ABI library loads and exports every symbol include/cudafoam.h
declares; without a device it fails loudly (CF_ERR_NO_DEVICE), never falls
back to the CPU."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(cf_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("cf_context_create", "cf_set_topology", "cf_set_coeffs", "cf_pcg",
                 "cf_bicgstab", "cf_delta", "cf_solve", "cf_solve_device", "cf_last_error"):
        assert must in names


def test_library_exports_all_declared_symbols():
    from metal4foam_b200 import _lib
    L = _lib.load()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, f"declared but not exported: {missing}"
    assert L.cf_abi_version() == 1


def test_signatures_cover_header():
    from metal4foam_b200 import _lib
    bound = {s[0] for s in _lib.SIGNATURES}
    assert set(declared_functions()) <= bound


def test_no_device_fails_loudly():
    from conftest import gpu_available
    if gpu_available():
        pytest.skip("a device is present")
    from metal4foam_b200 import _lib
    with pytest.raises(_lib.CudaFoamError) as ei:
        _lib.Context(0)
    assert ei.value.code in (5, 6)


def test_options_defaults():
    from metal4foam_b200 import _lib
    o = _lib.default_options()
    assert o.tolerance == 1e-6 and o.relTol == 0.0 and o.maxIter == 1000
    assert o.maxRestarts == 8 and o.iterationsPerSync == 1 and o.deflate == 0
    assert o.chebyshevOrder == 8 and o.chebyshevRatio == 30.0 and o.graph == 1


def test_solver_selection_and_errors():
    import numpy as np
    from metal4foam_b200 import mesh
    from metal4foam_b200.solver import FatalError, cudaPBiCGStab, cudaPCG, lduMatrix
    s = mesh.upwind3d((4, 4, 4))
    asym = lduMatrix(s.addr, s.diag, s.upper, s.lower)
    sym = lduMatrix(s.addr, s.diag, s.upper)
    assert isinstance(lduMatrix.solver.New("U", asym, {"solver": "cudaPBiCGStab"}), cudaPBiCGStab)
    assert isinstance(lduMatrix.solver.New("p", sym, {"solver": "cudaPCG"}), cudaPCG)
    with pytest.raises(FatalError):
        lduMatrix.solver.New("U", asym, {"solver": "cudaPCG"})
    with pytest.raises(FatalError):
        lduMatrix.solver.New("p", sym, {"solver": "cudaPCG", "cuda": {"bogus": 1}})
    solver = lduMatrix.solver.New("p", sym, {"solver": "cudaPCG"}, interfaces=[object()])
    with pytest.raises(FatalError):
        solver.solve(np.zeros(s.n), s.source)


def test_noalloc_rejects_null_pointers_before_any_device_work():
    """cf_ldu_spmv_dot_noalloc checks its pointers on the host: a NULL
    addressing array (read for every row with faces) or operand returns
    CF_ERR_INVALID_ARG and launches nothing, so this runs without a GPU.
    The pointer values below are never dereferenced."""
    from metal4foam_b200 import _lib
    L = _lib.load()
    fake = 0x1000
    args = [fake] * 9  # diag upper lower low upp ownStart losort losortStart x
    names = ["diag", "upper", "lower", "lowAddr", "uppAddr", "ownStartAddr", "losortAddr",
             "losortStartAddr", "x"]
    for k, name in enumerate(names):
        if name == "lower":   # NULL lower means symmetric
            continue
        a = list(args)
        a[k] = None
        rc = L.cf_ldu_spmv_dot_noalloc(10, *a, fake, fake, fake, None)
        assert rc == 1, name
        assert b"NULL" in L.cf_last_error(), name
    rc = L.cf_ldu_spmv_dot_noalloc(10, *args, fake, None, fake, None)   # y NULL
    assert rc == 1
    rc = L.cf_ldu_spmv_dot_noalloc(0, *args, fake, fake, fake, None)
    assert rc == 1
