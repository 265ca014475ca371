"""The oracle's kernel sequences (the checker of the fused-kernel tests)
against numpy restatements of the same element-wise FP32 expressions
(numpy float32 ufuncs round every product and sum separately, as the
reference kernels' source reads), on a small system.  CPU only."""
import numpy as np

from metal4foam_b200 import mesh

f = np.float32


def test_kernel_sequences_match_numpy_restatement(oracle):
    s = mesh.upwind3d((6, 5, 4), seed=9)
    seq = oracle.KernelSequence(s)
    n = s.n
    rng = np.random.default_rng(0)
    r, p0, v0, d, a0 = (rng.standard_normal(n).astype(f) for _ in range(5))
    al, be, om = f(0.37), f(0.81), f(1.13)
    rD = (1.0 / s.diag).astype(f)
    Af = seq.v
    # bicg_ab: p = r + beta (p0 - omega v0); y = rD p; AyA = A y
    out, sums = seq.bicg_ab(r, p0, v0, a0, float(be), float(om))
    p = r + be * (p0 - om * v0)
    y = rD * p
    assert np.array_equal(out["p"], p) and np.array_equal(out["yA"], y)
    assert np.array_equal(out["AyA"], Af.spmv(y)[0])
    assert sums[0] == np.dot(a0.astype(np.float64), out["AyA"].astype(np.float64))
    # bicg_cd: s = r - alpha AyA; z = rD s
    out, sums = seq.bicg_cd(r, v0, float(al))
    sv = r - al * v0
    assert np.array_equal(out["sA"], sv) and np.array_equal(out["zA"], rD * sv)
    assert sums[0] == np.sum(np.abs(sv.astype(np.float64)))
    # bicg_e: delta += (alpha y + omega z); r = s - omega t
    t = rng.standard_normal(n).astype(f)
    out, _ = seq.bicg_e(d, y, rD * sv, sv, t, a0, float(al), float(om))
    assert np.array_equal(out["deltaNext"], d + (al * y + om * (rD * sv)))
    assert np.array_equal(out["rAOut"], sv - om * t)
    # pcg: p = wA + beta p0; update with the Jacobi apply
    out, _ = seq.pcg_p_spmv(r, p0, float(be))
    assert np.array_equal(out["p"], r + be * p0)
    out, sums = seq.pcg_update(d, p0, r, v0, float(al), 1)
    rn = r - al * v0
    assert np.array_equal(out["deltaNext"], d + al * p0)
    assert np.array_equal(out["rAOut"], rn)
    assert np.array_equal(out["wAOut"], rn * rD)
    assert sums[1] == np.dot((rn * rD).astype(np.float64), rn.astype(np.float64))
