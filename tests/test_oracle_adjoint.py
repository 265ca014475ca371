"""Pins the FP64 CPU adjoint used as the reference of the GPU adjoint tests:
its forward and adjoint solutions agree with sparse direct FP64 solves
(scipy SuperLU) to 1e-10, and its gradients with the directly computed
ones, on the variable-coefficient Poisson problem (symmetric, one pinned
cell) and an asymmetric upwind problem."""
import numpy as np
import scipy.sparse.linalg as spla

from metal4foam_b200 import mesh


def rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def test_adjoint_reference_vs_direct_solves(oracle):
    cases = [mesh.adjoint_system((16, 15, 14), seed=51)]
    s = mesh.upwind3d((12, 11, 10), seed=52)
    cases.append((s, np.random.default_rng(53).standard_normal(s.n)))
    for s, xstar in cases:
        x, _ = oracle.cg64(s, tol=1e-13)
        lam, _ = oracle.cg64(s, b=x - xstar, tol=1e-10, transpose=True)
        lu = spla.splu(mesh.to_csr(s).tocsc())
        xd = lu.solve(s.source)
        ld = lu.solve(xd - xstar, trans="T")
        assert rel(x, xd) < 1e-10
        assert rel(lam, ld) < 1e-9
        got = oracle.face_gradients(s, lam, x)
        ref = oracle.face_gradients(s, ld, xd)
        for g, r in zip(got, ref):
            assert rel(g, r) < 1e-9
        # gradients by the dense formula dL/dA = -lambda x^T on the stored entries
        a = s.addr
        assert np.array_equal(got[0], -lam[a.lowerAddr] * x[a.upperAddr])
        assert np.array_equal(got[1], -lam[a.upperAddr] * x[a.lowerAddr])
        assert np.array_equal(got[2], -lam * x)
