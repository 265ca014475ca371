"""Decomposition into subdomains with processor interfaces (CPU).

The split system must be the original one: internal LDU matrices plus the
interface terms (row faceCells[k] gets -coeffs[k] * neighbour value, as
lduMatrix::Amul's updateMatrixInterfaces adds them) reproduce every row of
the unsplit A x; both sides of an interface list the same faces in the same
order; every face is either internal to one subdomain or on exactly one
interface pair."""
import numpy as np
import pytest

from metal4foam_b200 import decompose, mesh


CASES = {
    "varcoeff_slabs3": (lambda: mesh.varcoeff3d((9, 8, 7), seed=1, permute=False), "slab", 3),
    "varcoeff_random4": (lambda: mesh.varcoeff3d((8, 7, 6), seed=2, permute=True), "random", 4),
    "upwind_slabs2": (lambda: mesh.upwind3d((7, 6, 5), seed=3), "slab", 2),
    "poisson_random2": (lambda: mesh.poisson2d(13, 11, seed=4), "random", 2),
}


def partition(s, kind, k):
    if kind == "slab":
        return decompose.slab_partition(s.n, k)
    return np.random.default_rng(7).integers(0, k, s.n).astype(np.int32)


@pytest.mark.parametrize("name", sorted(CASES))
def test_interface_amul_equals_unsplit(oracle, name):
    make, kind, k = CASES[name]
    s = make()
    subs = decompose.decompose(s, partition(s, kind, k), k)
    x = np.random.default_rng(1).standard_normal(s.n)
    ys = decompose.interface_amul(subs, [x[sd.cells] for sd in subs], oracle.amul)
    y = decompose.assemble(subs, s.n, ys)
    ref = oracle.amul(s, x)
    assert np.allclose(y, ref, rtol=1e-13, atol=1e-13 * np.max(np.abs(ref)))


@pytest.mark.parametrize("name", sorted(CASES))
def test_faces_accounted_once_and_sides_match(name):
    make, kind, k = CASES[name]
    s = make()
    part = partition(s, kind, k)
    subs = decompose.decompose(s, part, k)
    assert sum(sd.n for sd in subs) == s.n
    seen = np.zeros(s.nf, np.int64)
    for sd in subs:
        for itf in sd.interfaces:
            other = next(i for i in subs[itf.neighbour].interfaces if i.neighbour == sd.rank)
            assert np.array_equal(itf.faces, other.faces)
            assert np.all(np.diff(itf.faces) > 0)
            seen[itf.faces] += 1
            # this side's cell is the face's owner or neighbour on this rank
            low, upp = s.addr.lowerAddr[itf.faces], s.addr.upperAddr[itf.faces]
            cell = sd.cells[itf.faceCells]
            assert np.all((cell == low) | (cell == upp))
            assert np.all(part[cell] == sd.rank)
    internal = sum(sd.system.nf for sd in subs)
    assert internal + np.count_nonzero(seen) == s.nf
    assert np.all((seen == 0) | (seen == 2))     # each interface face on both sides
    for sd in subs:
        a = sd.system.addr
        # local faces in LDU order (the C ABI validates it too)
        key = a.lowerAddr.astype(np.int64) * sd.n + a.upperAddr
        assert np.all(np.diff(key) > 0) and np.all(a.lowerAddr < a.upperAddr)


def test_single_subdomain_is_the_system():
    s = mesh.varcoeff3d((5, 4, 3), seed=5)
    (sd,) = decompose.decompose(s, np.zeros(s.n, np.int32), 1)
    assert not sd.interfaces and sd.n == s.n
    assert np.array_equal(sd.system.upper, s.upper)
    assert np.array_equal(sd.system.addr.lowerAddr, s.addr.lowerAddr)


def test_bad_partition_rejected():
    s = mesh.poisson2d(4, 4)
    with pytest.raises(ValueError):
        decompose.decompose(s, np.zeros(s.n, np.int32), 2)      # subdomain 1 empty
    with pytest.raises(ValueError):
        decompose.decompose(s, np.full(s.n, 3, np.int32), 2)
