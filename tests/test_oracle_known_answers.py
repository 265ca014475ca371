"""Known-answer tests that pin the CPU oracle where no reference test exists:
hand-checked LDU addressing, Amul, sumA, normFactor and checkConvergence
(OpenFOAM semantics the reference driver calls, metalFoamSolver.C:109-134),
plus internal consistency of the oracle's solvers."""
import numpy as np
import pytest

from metal4foam_b200 import mesh


def grid3x3():
    # 3x3 2-D grid, cells c = i + 3j; faces in LDU order (owner, neighbour)
    low, upp, _ = mesh.structured_faces((3, 3))
    return low, upp


def test_addressing_3x3_by_hand(oracle):
    low, upp = grid3x3()
    # faces sorted by owner then neighbour, written out by hand
    assert low.tolist() == [0, 0, 1, 1, 2, 3, 3, 4, 4, 5, 6, 7]
    assert upp.tolist() == [1, 3, 2, 4, 5, 4, 6, 5, 7, 8, 7, 8]
    a = mesh.ldu_addressing(9, low, upp)
    assert a.ownerStartAddr.tolist() == [0, 2, 4, 5, 7, 9, 10, 11, 12, 12]
    # faces grouped by neighbour, stable in face index
    assert a.losortAddr.tolist() == [0, 2, 1, 3, 5, 4, 7, 6, 8, 10, 9, 11]
    assert a.losortStartAddr.tolist() == [0, 0, 1, 2, 3, 5, 7, 8, 10, 12]
    own, los, losS = oracle.build_addressing(9, low, upp)
    assert np.array_equal(own, a.ownerStartAddr)
    assert np.array_equal(los, a.losortAddr)
    assert np.array_equal(losS, a.losortStartAddr)


def test_prism_faces_by_hand(oracle):
    """One layer of 2 x 1 quadrilaterals cut into triangles, two layers:
    cells ((k ny + j) nx + i) 2 + t; faces across each diagonal, between
    neighbouring quads (right edge of t0 to the left edge of the next
    quad's t1), and between the layers."""
    low, upp = mesh.prism_faces(2, 1, 2)
    pairs = sorted(zip(low.tolist(), upp.tolist()))
    want = sorted([(0, 1), (2, 3), (4, 5), (6, 7),          # diagonals
                   (0, 3), (4, 7),                          # quad (0,0) t0 | quad (1,0) t1
                   (0, 4), (1, 5), (2, 6), (3, 7)])         # layer 0 | layer 1
    assert pairs == want
    assert list(zip(low.tolist(), upp.tolist())) == want    # already in LDU order
    s = mesh.prism3d((9, 8, 7), seed=3)
    a = s.addr
    own, los, losS = oracle.build_addressing(s.n, a.lowerAddr, a.upperAddr)
    assert np.array_equal(own, a.ownerStartAddr)
    deg = np.bincount(a.lowerAddr, minlength=s.n) + np.bincount(a.upperAddr, minlength=s.n)
    assert deg.max() == 5 and s.n == 2 * 9 * 8 * 7
    assert s.nf == 9 * 8 * 7 + 8 * 8 * 7 + 9 * 7 * 7 + 2 * 9 * 8 * 6


def test_addressing_rejects_unsorted(oracle):
    low = np.array([0, 1, 0], np.int32)
    upp = np.array([1, 2, 2], np.int32)
    with pytest.raises(ValueError):
        oracle.build_addressing(3, low, upp)
    with pytest.raises(ValueError):
        mesh.ldu_addressing(3, low, upp)


def test_addressing_permuted_bit_exact(oracle):
    s = mesh.varcoeff3d((12, 10, 9), seed=7, permute=True)
    a = s.addr
    own, los, losS = oracle.build_addressing(s.n, a.lowerAddr, a.upperAddr)
    assert np.array_equal(own, a.ownerStartAddr)
    assert np.array_equal(los, a.losortAddr)
    assert np.array_equal(losS, a.losortStartAddr)
    # independent dense check: every face appears once, owner < neighbour
    pairs = set(zip(a.lowerAddr.tolist(), a.upperAddr.tolist()))
    assert len(pairs) == s.nf
    assert all(lo < hi for lo, hi in pairs)


def small_matrix():
    # 3 cells in a row, faces (0,1), (1,2)
    low = np.array([0, 1], np.int32)
    upp = np.array([1, 2], np.int32)
    addr = mesh.ldu_addressing(3, low, upp)
    diag = np.array([4.0, 5.0, 6.0])
    upper = np.array([-1.0, -2.0])
    lower = np.array([-0.5, -3.0])
    return mesh.LduSystem("k3", addr, diag, upper, lower, np.array([1.0, 2.0, 3.0]), np.zeros(3))


def test_amul_by_hand(oracle):
    s = small_matrix()
    # A = [[4, -1, 0], [-0.5, 5, -2], [0, -3, 6]]
    x = np.array([1.0, 2.0, 3.0])
    y = oracle.amul(s, x)
    assert y.tolist() == [4 - 2, -0.5 + 10 - 6, -6 + 18]
    yt = oracle.amul(s, x, transpose=True)
    assert yt.tolist() == [4 - 1, -1 + 10 - 9, -4 + 18]
    assert oracle.sumA(s).tolist() == [3.0, 2.5, 3.0]


def test_normfactor_constant_psi(oracle):
    s = small_matrix()
    psi = np.full(3, 2.0)
    Apsi = oracle.amul(s, psi)
    u = oracle.sumA(s)
    # A psi = xRef * u exactly, so only the source term remains
    nf = oracle.normfactor(psi, s.source, Apsi, u)
    expect = np.sum(np.abs(s.source - 2.0 * u)) + 1e-20
    assert nf == pytest.approx(expect, rel=0, abs=1e-15)


def test_check_convergence_edges(oracle):
    assert oracle.check_convergence(1e-6, 0.0, 1.0, 9.9e-7)
    assert not oracle.check_convergence(1e-6, 0.0, 1.0, 1e-6)      # strict <
    assert oracle.check_convergence(1e-9, 0.1, 1.0, 0.09)
    assert not oracle.check_convergence(1e-9, 0.1, 1.0, 0.1)
    assert not oracle.check_convergence(1e-30, 1e-21, 1.0, 1e-22)  # relTol below small_
    assert oracle.check_convergence(0.0, 1e-3, 2.0, 1.9e-3)


def test_amul_row_order_equals_face_loop(oracle):
    for s in (mesh.varcoeff3d((10, 9, 8), seed=3, permute=True), mesh.upwind3d((9, 8, 7), seed=4)):
        x = np.random.default_rng(0).standard_normal(s.n)
        y_face = oracle.amul(s, x)
        y_rows = oracle.amul_rows(s, x, nthreads=1)
        assert np.array_equal(y_face, y_rows)
        assert np.allclose(y_face, mesh.amul_numpy(s, x), rtol=1e-13, atol=1e-13)
        assert np.array_equal(oracle.amul(s, x, transpose=True),
                              oracle.amul_rows(s, x, transpose=True, nthreads=1))


def test_cheb_constants_recurrence(oracle):
    c = oracle.cheb_constants(4, 2.0, 30.0)
    beta, ratio = 2.0, 30.0
    alpha = beta / ratio
    theta, delta = 0.5 * (beta + alpha), 0.5 * (beta - alpha)
    sigma = theta / delta
    rho = 1 / sigma
    assert c[0] == np.float32(1 / theta)
    for i in range(1, 4):
        rn = 1 / (2 * sigma - rho)
        assert c[2 * i - 1] == np.float32(rn * rho)
        assert c[2 * i] == np.float32(2 * rn / delta)
        rho = rn


def test_cg64_accuracy(oracle):
    s = mesh.varcoeff3d((16, 16, 16), seed=2, permute=True)
    x, it = oracle.cg64(s, tol=1e-12)
    r = s.source - mesh.amul_numpy(s, x)
    assert np.linalg.norm(r) <= 2e-12 * np.linalg.norm(s.source)


def test_metal_emulation_poisson2d(oracle):
    s = mesh.poisson2d(64, 64, seed=1)
    r = oracle.metal_solve(s, chebyshevOrder=4, maxRestarts=4)
    assert r.deflated and r.converged and r.finalResidual < 1e-6
    x, _ = oracle.cg64(s)
    assert np.max(np.abs(r.psi - x)) < 1e-3 * np.max(np.abs(x))


def test_foam_pcg_dic_beats_diagonal(oracle):
    s = mesh.poisson2d(48, 48, seed=2)
    _, dic = oracle.foam_pcg(s, "DIC")
    _, dia = oracle.foam_pcg(s, "diagonal")
    assert dic.converged and dia.converged
    assert dic.nIterations < dia.nIterations


def test_metal_bicgstab_upwind(oracle):
    s = mesh.upwind3d((16, 16, 16), seed=5)
    r = oracle.metal_solve(s, bicgstab=True, tolerance=1e-8)
    assert r.converged and not r.deflated
    _, p = oracle.foam_pbicgstab(s, tolerance=1e-8)
    assert p.converged
