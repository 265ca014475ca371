"""Pins the oracle's restatement of the reference kernels against golden
vectors produced by the reference's own kernel source
(src/metal4Foam/shaders/metalFoamKernels.metal, compiled unchanged for the
CPU; tests/golden/make_golden.py).  Every kernel must match bit for bit."""
import ctypes as C
import os

import numpy as np
import pytest

from metal4foam_b200 import mesh

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "msl_kernels.npz")


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


def systems():
    return {"upwind": mesh.upwind3d((9, 8, 7), seed=21),
            "varperm": mesh.varcoeff3d((10, 9, 8), seed=22, permute=True)}


def eq(a, b):
    return np.array_equal(np.asarray(a).view(np.uint32), np.asarray(b).view(np.uint32))


@pytest.mark.parametrize("tag", ["upwind", "varperm"])
def test_restated_kernels_match_reference_kernels(oracle, gold, tag):
    L = oracle.lib()
    s = systems()[tag]
    n = s.n
    ng = (n + 255) // 256
    g = lambda k: gold[f"{tag}/{k}"]  # noqa: E731
    i = lambda k: np.array(gold[f"{tag}/in/{k}"])  # noqa: E731
    view = oracle.Ldu32View(s)
    part = np.zeros(ng, np.float32)
    y = np.zeros(n, np.float32)
    L.orc_k_ldu_spmv_dotw(C.byref(view.s), i("x"), i("w"), y, part)
    assert eq(y, g("spmv_dotw/y")) and eq(part, g("spmv_dotw/partials"))
    y2 = np.zeros(n, np.float32)
    L.orc_k_ldu_spmv(C.byref(view.s), i("x"), y2)
    assert eq(y2, g("spmv/y"))
    w = np.zeros(n, np.float32)
    z = np.zeros(n, np.float32)
    L.orc_k_cheb_init(n, i("r"), i("rD"), w, z, np.float32(0.7))
    assert eq(w, g("cheb_init/w")) and eq(z, g("cheb_init/z"))
    L.orc_k_cheb_step(n, i("r"), i("v"), i("rD"), w, z, np.float32(0.3), np.float32(1.1))
    assert eq(w, g("cheb_step/w")) and eq(z, g("cheb_step/z"))
    e = np.zeros(n, np.float32)
    L.orc_k_emul(n, i("rD"), i("p0"), e)
    assert eq(e, g("emul/out"))
    wa = np.zeros(n, np.float32)
    L.orc_k_pcg_precond_dot(n, i("r"), i("rD"), wa, part)
    assert eq(wa, g("precond_dot/wA")) and eq(part, g("precond_dot/partials"))
    p = i("p0")
    L.orc_k_pcg_update_p(n, p, i("wA"), i("s16"))
    assert eq(p, g("update_p/p"))
    d, r = i("dl"), i("r")
    L.orc_k_pcg_update_sol_res(n, d, r, i("p0"), i("wA"), i("s16"), part)
    assert eq(d, g("update_sol_res/delta")) and eq(r, g("update_sol_res/rA"))
    assert eq(part, g("update_sol_res/partials"))
    L.orc_k_dot_partial(n, i("x"), i("w"), part)
    assert eq(part, g("dot_partial/partials"))
    p = i("p0")
    L.orc_k_bicg_update_p(n, p, i("r"), i("AyA"), i("s16"))
    assert eq(p, g("bicg_update_p/p"))
    sa = np.zeros(n, np.float32)
    L.orc_k_bicg_s_res(n, sa, i("r"), i("AyA"), i("s16"), part)
    assert eq(sa, g("bicg_s_res/sA")) and eq(part, g("bicg_s_res/partials"))
    d = i("dl")
    L.orc_k_bicg_early_update(n, d, i("yA"), i("s16"))
    assert eq(d, g("bicg_early_update/delta"))
    d, r = i("dl"), i("r")
    L.orc_k_bicg_update_sol_res(n, d, i("yA"), i("zA"), r, i("sA"), i("tA"), i("s16"), part)
    assert eq(d, g("bicg_update_sol_res/delta")) and eq(r, g("bicg_update_sol_res/rA"))
    assert eq(part, g("bicg_update_sol_res/partials"))


@pytest.mark.parametrize("count", [2, 37, 300])
def test_restated_reduce_scalars_matches_reference(oracle, gold, count):
    L = oracle.lib()
    P1 = np.array(gold[f"reduce/{count}/P1"])
    P2 = np.array(gold[f"reduce/{count}/P2"])
    for mode in range(6):
        for first in (0, 1):
            s = np.array(gold[f"reduce/{count}/{mode}/{first}/s_in"])
            L.orc_k_reduce_scalars(P1, P2, s, count, mode, first)
            assert eq(s, gold[f"reduce/{count}/{mode}/{first}/s_out"]), (mode, first)


def test_live_reference_kernels_random_inputs(oracle):
    """When the compiled reference kernels are present, compare on fresh
    seeded inputs too (covers sizes the fixtures do not)."""
    ref = oracle.ref_lib()
    if ref is None:
        pytest.skip("oracle/_ref not built here")
    P = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    for s in (mesh.poisson2d(31, 17, seed=3), mesh.upwind3d((11, 7, 5), seed=4)):
        n = s.n
        view = oracle.Ldu32View(s)
        a = s.addr
        addr = [np.ascontiguousarray(x, np.uint32) for x in a.arrays()]
        rng = np.random.default_rng(n)
        x = rng.standard_normal(n).astype(np.float32)
        w = rng.standard_normal(n).astype(np.float32)
        ng = (n + 255) // 256
        y1, p1 = np.zeros(n, np.float32), np.zeros(ng, np.float32)
        y2, p2 = np.zeros(n, np.float32), np.zeros(ng, np.float32)
        ref.ref_ldu_spmv_dotw(n, P(view.diag), P(view.upper), P(view.lower), *map(P, addr),
                              P(x), P(w), P(y1), P(p1))
        oracle.lib().orc_k_ldu_spmv_dotw(C.byref(view.s), x, w, y2, p2)
        assert eq(y1, y2) and eq(p1, p2)
