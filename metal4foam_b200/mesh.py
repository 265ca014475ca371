"""Seeded synthetic LDU systems and OpenFOAM ``lduAddressing`` construction.

An OpenFOAM ``lduMatrix`` stores a square sparse matrix as

* ``diag[n]`` -- the diagonal,
* ``upper[nf]`` -- ``A[l(f), u(f)]`` for every internal face ``f``,
* ``lower[nf]`` -- ``A[u(f), l(f)]`` (aliased to ``upper`` when symmetric),

with ``l = lowerAddr`` (owner) and ``u = upperAddr`` (neighbour), faces in
upper-triangular order: ``l(f) < u(f)``, sorted by owner and then by
neighbour.  ``lduAddressing`` derives three more arrays from that
(the reference's kernels consume all five,
src/metal4Foam/shaders/metalFoamKernels.metal:64-109, and its backend
uploads them once per mesh, src/metal4Foam/backend/metalFoamBackend.C:454-519):

* ``ownerStartAddr[n+1]`` -- first face owned by each cell, ``[n] = nf``;
* ``losortAddr[nf]`` -- face indices ordered by neighbour, stable in face
  index;
* ``losortStartAddr[n+1]`` -- first ``losort`` slot of each neighbour cell,
  ``[n] = nf``.

The construction here is sort-based (numpy); the oracle builds the same
arrays by counting sort in C, and the tests require the two to agree bit
for bit.

The generators produce the five workloads the solver is measured on
(2-D Poisson 128^2, permuted variable-coefficient 128^3, upwind
convection-diffusion 96^3, a batch of 48 uneven meshes plus a 64^3
three-component momentum matrix, and the 64^3 adjoint problem).  Every
array is drawn from ``numpy.random.default_rng(seed)`` in a fixed order so
the same seed always gives the same system.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

__all__ = [
    "LduAddressing",
    "LduSystem",
    "ldu_addressing",
    "structured_faces",
    "poisson2d",
    "varcoeff3d",
    "upwind3d",
    "batched_systems",
    "momentum_multi_rhs",
    "adjoint_system",
    "to_csr",
    "amul_numpy",
    "permute_cells",
]


@dataclass
class LduAddressing:
    """The five int32 arrays of OpenFOAM's ``lduAddressing``."""

    n: int
    nf: int
    lowerAddr: np.ndarray
    upperAddr: np.ndarray
    ownerStartAddr: np.ndarray
    losortAddr: np.ndarray
    losortStartAddr: np.ndarray

    def arrays(self):
        return (self.lowerAddr, self.upperAddr, self.ownerStartAddr,
                self.losortAddr, self.losortStartAddr)


@dataclass
class LduSystem:
    """One linear system ``A psi = source`` in LDU form (FP64 coefficients)."""

    name: str
    addr: LduAddressing
    diag: np.ndarray
    upper: np.ndarray
    lower: Optional[np.ndarray]          # None: symmetric (lower == upper)
    source: np.ndarray
    psi: np.ndarray
    meta: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return self.addr.n

    @property
    def nf(self) -> int:
        return self.addr.nf

    @property
    def symmetric(self) -> bool:
        return self.lower is None

    @property
    def lower_or_upper(self) -> np.ndarray:
        return self.upper if self.lower is None else self.lower


def ldu_addressing(n: int, low: np.ndarray, upp: np.ndarray) -> LduAddressing:
    """Build ownerStart/losort/losortStart from owner/neighbour arrays.

    ``low``/``upp`` must already be in LDU order (owner < neighbour, sorted by
    owner then neighbour); this is checked.
    """
    low = np.ascontiguousarray(low, dtype=np.int32)
    upp = np.ascontiguousarray(upp, dtype=np.int32)
    nf = low.shape[0]
    if upp.shape[0] != nf:
        raise ValueError("lowerAddr and upperAddr differ in length")
    if nf:
        if low.min() < 0 or upp.max() >= n:
            raise ValueError("face addressing out of range")
        if np.any(low >= upp):
            raise ValueError("faces must satisfy owner < neighbour")
        key = low.astype(np.int64) * n + upp
        if np.any(np.diff(key) <= 0):
            raise ValueError("faces must be sorted by owner, then neighbour")
    own_counts = np.bincount(low, minlength=n)
    own_start = np.zeros(n + 1, dtype=np.int32)
    np.cumsum(own_counts, out=own_start[1:])
    losort = np.argsort(upp, kind="stable").astype(np.int32)
    nbr_counts = np.bincount(upp, minlength=n)
    losort_start = np.zeros(n + 1, dtype=np.int32)
    np.cumsum(nbr_counts, out=losort_start[1:])
    return LduAddressing(n, nf, low, upp, own_start, losort, losort_start)


def structured_faces(dims: Sequence[int]):
    """Internal faces of an nx x ny (x nz) structured grid in LDU order.

    Cell index ``c = i + nx*(j + ny*k)``.  Returns ``(low, upp, axis)`` with
    ``axis[f]`` the grid direction of face ``f``.
    """
    dims = tuple(int(d) for d in dims)
    n = int(np.prod(dims))
    idx = np.arange(n, dtype=np.int64).reshape(dims[::-1])  # [k][j][i]
    lows, upps, axes = [], [], []
    nd = len(dims)
    for d in range(nd):
        ax = nd - 1 - d                     # numpy axis of grid direction d
        sl_lo = [slice(None)] * nd
        sl_hi = [slice(None)] * nd
        sl_lo[ax] = slice(0, dims[d] - 1)
        sl_hi[ax] = slice(1, dims[d])
        lo = idx[tuple(sl_lo)].ravel()
        hi = idx[tuple(sl_hi)].ravel()
        lows.append(lo)
        upps.append(hi)
        axes.append(np.full(lo.shape, d, dtype=np.int8))
    low = np.concatenate(lows)
    upp = np.concatenate(upps)
    axis = np.concatenate(axes)
    order = np.lexsort((upp, low))
    return (low[order].astype(np.int32), upp[order].astype(np.int32),
            axis[order])


def _rowsum_abs_offdiag(n, low, upp, upper, lower):
    s = np.zeros(n)
    np.add.at(s, low, np.abs(upper))
    np.add.at(s, upp, np.abs(lower))
    return s


def _bincount_sum(n, idx, w):
    return np.bincount(idx, weights=w, minlength=n)


def permute_cells(newlabel: np.ndarray, low, upp, *face_arrays):
    """Relabel cells (old c -> newlabel[c]) and re-sort faces into LDU order.

    Face arrays travel with their faces.  Faces whose orientation flips swap
    nothing here: callers pass symmetric coefficients only.
    """
    a = newlabel[low]
    b = newlabel[upp]
    lo = np.minimum(a, b).astype(np.int32)
    hi = np.maximum(a, b).astype(np.int32)
    order = np.lexsort((hi, lo))
    out = [lo[order], hi[order]]
    for arr in face_arrays:
        out.append(arr[order])
    return out


def relabel(sysm: LduSystem, seed: int) -> LduSystem:
    """The same linear system with cells renumbered by a seeded permutation
    (faces re-oriented and re-sorted into LDU order; an asymmetric face whose
    owner and neighbour swap also swaps its upper/lower coefficients)."""
    rng = np.random.default_rng(seed)
    nl = rng.permutation(sysm.n)
    a = sysm.addr
    lo = nl[a.lowerAddr]
    hi = nl[a.upperAddr]
    swap = lo > hi
    lower = sysm.lower_or_upper
    up = np.where(swap, lower, sysm.upper)
    lw = np.where(swap, sysm.upper, lower)
    L = np.minimum(lo, hi)
    H = np.maximum(lo, hi)
    o = np.lexsort((H, L))
    addr = ldu_addressing(sysm.n, L[o], H[o])
    diag = np.empty(sysm.n)
    diag[nl] = sysm.diag
    src = np.empty(sysm.n)
    src[nl] = sysm.source
    psi = np.empty(sysm.n)
    psi[nl] = sysm.psi
    return LduSystem(sysm.name + f"_relabel{seed}", addr, diag, up[o],
                     None if sysm.lower is None else lw[o], src, psi, dict(sysm.meta))


def poisson2d(nx: int = 128, ny: int = 128, seed: int = 0) -> LduSystem:
    """2-D 5-point Neumann Poisson with setReference on cell 0.

    upper = lower = -1, diag = number of neighbours, diag[0] doubled;
    source ~ N(0,1) projected to zero mean; psi0 = 0.
    """
    low, upp, _ = structured_faces((nx, ny))
    n = nx * ny
    addr = ldu_addressing(n, low, upp)
    upper = -np.ones(addr.nf)
    diag = (np.bincount(low, minlength=n) + np.bincount(upp, minlength=n)).astype(np.float64)
    diag[0] *= 2.0                                   # setReference(0, 0)
    rng = np.random.default_rng(seed)
    b = rng.standard_normal(n)
    b -= b.mean()
    return LduSystem(f"poisson2d_{nx}x{ny}", addr, diag, upper, None, b,
                     np.zeros(n), dict(dims=(nx, ny), seed=seed))


def _varcoeff_coeffs(low, upp, k):
    ka = k[low]
    kb = k[upp]
    return -2.0 * ka * kb / (ka + kb)


def varcoeff3d(dims=(128, 128, 128), seed: int = 1, permute: bool = True,
               reference_cell: bool = True) -> LduSystem:
    """Variable-coefficient pressure matrix on a structured grid.

    k ~ 10**U(-2, 2) per cell; face coefficient = -harmonic mean of the two
    cells' k; diag = -sum(off-diagonals); Neumann boundaries; setReference on
    cell 0 (diag doubled).  With ``permute`` the cells are relabelled by a
    seeded random permutation and the faces re-sorted into LDU order.
    source ~ N(0,1), zero mean; psi0 = 0.  ``dims`` may be 2-D or 3-D.
    """
    dims = tuple(int(d) for d in dims)
    n = int(np.prod(dims))
    rng = np.random.default_rng(seed)
    k = 10.0 ** rng.uniform(-2.0, 2.0, n)
    low, upp, _ = structured_faces(dims)
    coef = _varcoeff_coeffs(low, upp, k)
    if permute:
        newlabel = rng.permutation(n).astype(np.int64)
        low, upp, coef = permute_cells(newlabel, low, upp, coef)
    addr = ldu_addressing(n, low, upp)
    diag = -(_bincount_sum(n, addr.lowerAddr, coef) + _bincount_sum(n, addr.upperAddr, coef))
    if reference_cell:
        diag[0] *= 2.0
    b = rng.standard_normal(n)
    b -= b.mean()
    name = "varcoeff3d_" + "x".join(map(str, dims)) + ("_perm" if permute else "")
    return LduSystem(name, addr, diag, coef, None, b, np.zeros(n),
                     dict(dims=dims, seed=seed, permute=permute))


def prism_faces(nx: int, ny: int, nz: int):
    """Internal faces of an extruded triangulated grid in LDU order: each of
    the nx x ny quadrilaterals of a layer is cut along its diagonal into two
    triangles, and nz layers are stacked, so an interior cell (a triangular
    prism) has five neighbours (three lateral, two axial).  Cell of quad
    (i, j), triangle t (0: below the diagonal, 1: above), layer k:
    ((k ny + j) nx + i) 2 + t."""
    def cid(i, j, k, t):
        return ((k * ny + j) * nx + i) * 2 + t
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    pairs = [(cid(i, j, k, 0), cid(i, j, k, 1))]               # across the diagonal
    m = i + 1 < nx
    pairs.append((cid(i[m], j[m], k[m], 0), cid(i[m] + 1, j[m], k[m], 1)))
    m = j + 1 < ny
    pairs.append((cid(i[m], j[m], k[m], 1), cid(i[m], j[m] + 1, k[m], 0)))
    for t in (0, 1):
        m = k + 1 < nz
        pairs.append((cid(i[m], j[m], k[m], t), cid(i[m], j[m], k[m] + 1, t)))
    a = np.concatenate([p[0] for p in pairs]).astype(np.int64)
    b = np.concatenate([p[1] for p in pairs]).astype(np.int64)
    low, upp = np.minimum(a, b), np.maximum(a, b)
    order = np.lexsort((upp, low))
    return low[order].astype(np.int32), upp[order].astype(np.int32)


def prism3d(dims=(24, 24, 16), seed: int = 6, permute: bool = True) -> LduSystem:
    """Variable-coefficient pressure matrix on triangular prisms (five
    neighbours per interior cell, see prism_faces): coefficients, reference
    cell and source as varcoeff3d; ``dims`` = (nx, ny, nz) quadrilaterals
    per layer and layers, 2 nx ny nz cells."""
    nx, ny, nz = (int(d) for d in dims)
    n = 2 * nx * ny * nz
    rng = np.random.default_rng(seed)
    k = 10.0 ** rng.uniform(-2.0, 2.0, n)
    low, upp = prism_faces(nx, ny, nz)
    coef = _varcoeff_coeffs(low, upp, k)
    if permute:
        newlabel = rng.permutation(n).astype(np.int64)
        low, upp, coef = permute_cells(newlabel, low, upp, coef)
    addr = ldu_addressing(n, low, upp)
    diag = -(_bincount_sum(n, addr.lowerAddr, coef) + _bincount_sum(n, addr.upperAddr, coef))
    diag[0] *= 2.0
    b = rng.standard_normal(n)
    b -= b.mean()
    name = f"prism3d_{nx}x{ny}x{nz}" + ("_perm" if permute else "")
    return LduSystem(name, addr, diag, coef, None, b, np.zeros(n),
                     dict(dims=(nx, ny, nz), seed=seed, permute=permute))


def _fourier_velocity(rng, nmodes=8):
    ks = rng.integers(-3, 4, size=(nmodes, 3)).astype(np.float64)
    phases = rng.uniform(0.0, 2.0 * np.pi, nmodes)
    amps = rng.standard_normal((nmodes, 3))
    amps /= np.linalg.norm(amps, axis=1, keepdims=True)

    def u(x):                               # x: (m, 3) in [0,1]^3 -> (m, 3)
        arg = 2.0 * np.pi * (x @ ks.T) + phases   # (m, nmodes)
        return np.cos(arg) @ amps
    return u


def upwind3d(dims=(96, 96, 96), seed: int = 2, D: float = 0.05) -> LduSystem:
    """First-order upwind convection-diffusion (asymmetric).

    Velocity u = sum of 8 seeded Fourier modes of unit amplitude on the unit
    cube; face flux F = u(x_face) . n_face with n pointing owner->neighbour;
    lower = -(D + max(F, 0)), upper = -(D + max(-F, 0)),
    diag = sum |off-diagonals of the row| + 0.01; source ~ U(-1, 1); psi0 = 0.
    """
    dims = tuple(int(d) for d in dims)
    if len(dims) == 2:
        dims3 = dims + (1,)
    else:
        dims3 = dims
    n = int(np.prod(dims))
    rng = np.random.default_rng(seed)
    ufield = _fourier_velocity(rng)
    low, upp, axis = structured_faces(dims)
    nx, ny, _ = dims3
    i = low % nx
    j = (low // nx) % ny
    kk = low // (nx * ny)
    h = np.array([1.0 / d for d in dims3])
    xc = np.stack([(i + 0.5) * h[0], (j + 0.5) * h[1], (kk + 0.5) * h[2]], axis=1)
    xc[np.arange(len(low)), axis] += 0.5 * h[axis]
    F = ufield(xc)[np.arange(len(low)), axis]
    lower = -(D + np.maximum(F, 0.0))
    upper = -(D + np.maximum(-F, 0.0))
    addr = ldu_addressing(n, low, upp)
    diag = _rowsum_abs_offdiag(n, low, upp, upper, lower) + 0.01
    b = rng.uniform(-1.0, 1.0, n)
    return LduSystem("upwind3d_" + "x".join(map(str, dims)), addr, diag, upper,
                     lower, b, np.zeros(n), dict(dims=dims, seed=seed, D=D))


def batched_systems(count: int = 48, seed: int = 3, nmin: float = 1e3,
                    nmax: float = 1e6):
    """Independent pressure systems with log-uniform cell counts.

    Each system is 2-D or 3-D (seeded), per-axis dimensions drawn from the
    seed so the cell count is about 10**U(log10 nmin, log10 nmax); the
    coefficients are generated as in :func:`varcoeff3d` without permutation.
    """
    rng = np.random.default_rng(seed)
    out = []
    for s in range(count):
        nd = int(rng.integers(2, 4))
        target = 10.0 ** rng.uniform(np.log10(nmin), np.log10(nmax))
        if nd == 2:
            r = 2.0 ** rng.uniform(-1.0, 1.0)
            nx = max(2, int(round(np.sqrt(target * r))))
            ny = max(2, int(round(target / nx)))
            dims = (nx, ny)
        else:
            base = target ** (1.0 / 3.0)
            nx = max(2, int(round(base * 2.0 ** rng.uniform(-0.5, 0.5))))
            ny = max(2, int(round(base * 2.0 ** rng.uniform(-0.5, 0.5))))
            nz = max(2, int(round(target / (nx * ny))))
            dims = (nx, ny, nz)
        sub = int(rng.integers(0, 2**31 - 1))
        sysm = varcoeff3d(dims, seed=sub, permute=False)
        sysm.name = f"batch{s:02d}_" + sysm.name
        out.append(sysm)
    return out


def momentum_multi_rhs(dims=(64, 64, 64), seed: int = 4, nrhs: int = 3):
    """One asymmetric momentum matrix (upwind, as :func:`upwind3d`) with
    ``nrhs`` right-hand sides ~ N(0,1) (Ux, Uy, Uz sharing one matrix)."""
    sysm = upwind3d(dims, seed=seed)
    rng = np.random.default_rng(seed + 1000)
    rhs = rng.standard_normal((nrhs, sysm.n))
    return sysm, rhs


def adjoint_system(dims=(64, 64, 64), seed: int = 5):
    """Variable-coefficient Poisson (unpermuted) plus a target x* ~ N(0,1)
    for the loss L = 0.5*||x - x*||^2."""
    sysm = varcoeff3d(dims, seed=seed, permute=False)
    rng = np.random.default_rng(seed + 1000)
    xstar = rng.standard_normal(sysm.n)
    return sysm, xstar


def to_csr(sysm: LduSystem):
    """scipy.sparse CSR matrix of an LDU system (test helper)."""
    import scipy.sparse as sp
    a = sysm.addr
    lo = sysm.lower_or_upper
    rows = np.concatenate([np.arange(a.n), a.lowerAddr, a.upperAddr])
    cols = np.concatenate([np.arange(a.n), a.upperAddr, a.lowerAddr])
    vals = np.concatenate([sysm.diag, sysm.upper, lo])
    return sp.csr_matrix((vals, (rows, cols)), shape=(a.n, a.n))


def amul_numpy(sysm: LduSystem, x: np.ndarray) -> np.ndarray:
    """y = A x (FP64, numpy, order-insensitive; test helper)."""
    a = sysm.addr
    y = sysm.diag * x
    y += np.bincount(a.lowerAddr, weights=sysm.upper * x[a.upperAddr], minlength=a.n)
    y += np.bincount(a.upperAddr, weights=sysm.lower_or_upper * x[a.lowerAddr], minlength=a.n)
    return y
