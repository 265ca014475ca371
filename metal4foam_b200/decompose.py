"""Decomposition of one LDU system into subdomains with processor interfaces.

OpenFOAM's decomposePar splits a mesh into processor meshes; each keeps its
own cells and internal faces and turns every face whose two cells went to
different processors into a face of a processor patch.  The matrix of a
processor mesh is then its own LDU matrix plus, per processor patch, the
face-cells and interface coefficients through which
lduMatrix::Amul's updateMatrixInterfaces couples it to the neighbour:
row faceCells[k] gets -interfaceBouCoeffs[k] * psi_neighbour[k].

:func:`decompose` does the same on an :class:`~metal4foam_b200.mesh.LduSystem`
given a cell-to-subdomain map.  Cells keep their relative order, so every
subdomain's faces stay in LDU order; the faces of an interface are listed
in global face order on both sides, so face k of subdomain a's interface to
b is face k of b's interface to a.  The coupled system is the original one:
for a face f split between owner cell o (on a) and neighbour cell q (on b),
a's row o gets upper[f] * psi_q and b's row q gets lower[f] * psi_o, so the
interface coefficients are -upper[f] on a's side and -lower[f] on b's.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List

import numpy as np

from .mesh import LduSystem, ldu_addressing


@dataclass
class Interface:
    neighbour: int              # subdomain across the interface
    faceCells: np.ndarray       # int32, this side's local cells, global face order
    coeffs: np.ndarray          # FP64 interfaceBouCoeffs
    faces: np.ndarray           # int64, the global faces (for checks)


@dataclass
class Subdomain:
    rank: int
    cells: np.ndarray           # global cell of each local cell (ascending)
    system: LduSystem           # internal matrix, source and psi of the local cells
    interfaces: List[Interface]

    @property
    def n(self) -> int:
        return self.system.n

    def interface_arrays(self):
        """(neighbour, nFaces, faceCells, coeffs) as the C ABI takes them."""
        nb = np.array([i.neighbour for i in self.interfaces], np.int32)
        nfc = np.array([len(i.faceCells) for i in self.interfaces], np.int32)
        fc = (np.concatenate([i.faceCells for i in self.interfaces]).astype(np.int32)
              if self.interfaces else np.zeros(0, np.int32))
        cf = (np.concatenate([i.coeffs for i in self.interfaces])
              if self.interfaces else np.zeros(0))
        return nb, nfc, np.ascontiguousarray(fc), np.ascontiguousarray(cf, np.float64)


def slab_partition(n: int, nparts: int) -> np.ndarray:
    """Cells split into nparts consecutive index ranges (geometric slabs of a
    structured mesh numbered x fastest)."""
    return np.minimum((np.arange(n, dtype=np.int64) * nparts) // max(n, 1),
                      nparts - 1).astype(np.int32)


def decompose(sysm: LduSystem, part: np.ndarray, nparts: int) -> List[Subdomain]:
    part = np.asarray(part, np.int32)
    if part.shape != (sysm.n,) or part.min() < 0 or part.max() >= nparts:
        raise ValueError("part must map every cell to a subdomain in [0, nparts)")
    a = sysm.addr
    low = a.lowerAddr.astype(np.int64)
    upp = a.upperAddr.astype(np.int64)
    lower = sysm.lower_or_upper
    pl, pu = part[low], part[upp]
    loc = np.empty(sysm.n, np.int64)
    out = []
    for r in range(nparts):
        cells = np.flatnonzero(part == r)
        if cells.size == 0:
            raise ValueError(f"subdomain {r} has no cells")
        loc[cells] = np.arange(cells.size)
        inner = np.flatnonzero((pl == r) & (pu == r))
        addr = ldu_addressing(cells.size, loc[low[inner]], loc[upp[inner]])
        sub = LduSystem(name=f"{sysm.name}_p{r}", addr=addr,
                        diag=np.ascontiguousarray(sysm.diag[cells]),
                        upper=np.ascontiguousarray(sysm.upper[inner]),
                        lower=None if sysm.lower is None
                        else np.ascontiguousarray(sysm.lower[inner]),
                        source=np.ascontiguousarray(sysm.source[cells]),
                        psi=np.ascontiguousarray(sysm.psi[cells]))
        ifaces = []
        for q in range(nparts):
            if q == r:
                continue
            own_side = np.flatnonzero((pl == r) & (pu == q))    # r holds the owner
            nbr_side = np.flatnonzero((pl == q) & (pu == r))    # r holds the neighbour
            faces = np.sort(np.concatenate([own_side, nbr_side]))
            if faces.size == 0:
                continue
            is_owner = pl[faces] == r
            fcell = np.where(is_owner, low[faces], upp[faces])
            coeff = np.where(is_owner, -sysm.upper[faces], -lower[faces])
            ifaces.append(Interface(q, loc[fcell].astype(np.int32), coeff.astype(np.float64),
                                    faces))
        out.append(Subdomain(r, cells, sub, ifaces))
    return out


def assemble(subs: List[Subdomain], n: int, local: List[np.ndarray]) -> np.ndarray:
    """Scatter per-subdomain fields back into one global field."""
    x = np.empty(n)
    for s, v in zip(subs, local):
        x[s.cells] = v
    return x


def interface_amul(subs: List[Subdomain], xs: List[np.ndarray], amul_local) -> List[np.ndarray]:
    """A x per subdomain with the interface terms (host reference used by the
    tests): amul_local(system, x) is the internal product, then every row
    faceCells[k] gets -coeffs[k] * (neighbour's x across face k)."""
    ys = []
    for s, x in zip(subs, xs):
        y = amul_local(s.system, x)
        for itf in s.interfaces:
            other = subs[itf.neighbour]
            back = next(i for i in other.interfaces if i.neighbour == s.rank)
            halo = xs[itf.neighbour][back.faceCells]
            for k in range(len(itf.faceCells)):
                y[itf.faceCells[k]] -= itf.coeffs[k] * halo[k]
        ys.append(y)
    return ys
