"""The plugin surface of the reference, mirrored for the host side.

metal4Foam registers two ``lduMatrix::solver`` subclasses, selected by name
from an fvSolution dictionary (src/metal4Foam/solvers/metalPCG.C:16-19,
src/metal4Foam/solvers/metalPBiCGStab.C:16-22) and sharing one FP64 driver
(src/metal4Foam/solvers/metalFoamSolver.C:77-437).  This module keeps that
shape -- the same class roles, names and argument meaning, the same
controls and the same error behaviour -- over the C ABI of libcudafoam.so,
under the run-time names ``cudaPCG`` and ``cudaPBiCGStab``:

    matrix = lduMatrix(addressing, diag, upper, lower=None)
    solver = lduMatrix.solver.New("p", matrix, {"solver": "cudaPCG",
                                                "tolerance": 1e-6,
                                                "cuda": {"maxRestarts": 4}})
    perf = solver.solve(psi, source)      # psi updated in place

The compiled OpenFOAM adapter with the same behaviour lives in
``metal4foam_b200/openfoam`` (built with wmake where OpenFOAM exists).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, Optional

import numpy as np

from . import _lib
from .mesh import LduAddressing, ldu_addressing

__all__ = ["FatalError", "lduAddressing", "lduMatrix", "solverPerformance", "cudaFoamSolver",
           "cudaPCG", "cudaPBiCGStab", "backend_cache_clear"]


class FatalError(RuntimeError):
    """OpenFOAM's FatalError: the run cannot continue."""


class lduAddressing:
    """Accessors of OpenFOAM's lduAddressing over :class:`mesh.LduAddressing`."""

    def __init__(self, addr: LduAddressing):
        self._a = addr

    @classmethod
    def from_faces(cls, nCells, lowerAddr, upperAddr):
        return cls(ldu_addressing(int(nCells), lowerAddr, upperAddr))

    def size(self):
        return self._a.n

    def lowerAddr(self):
        return self._a.lowerAddr

    def upperAddr(self):
        return self._a.upperAddr

    def ownerStartAddr(self):
        return self._a.ownerStartAddr

    def losortAddr(self):
        return self._a.losortAddr

    def losortStartAddr(self):
        return self._a.losortStartAddr


class lduMatrix:
    """FP64 LDU coefficients on an addressing (lower None: symmetric)."""

    solver = None  # set below to the run-time selection front end

    def __init__(self, addressing, diag, upper, lower=None, interfaces=None):
        if isinstance(addressing, LduAddressing):
            addressing = lduAddressing(addressing)
        self._addr = addressing
        self._diag = np.ascontiguousarray(diag, np.float64)
        self._upper = np.ascontiguousarray(upper, np.float64)
        self._lower = None if lower is None else np.ascontiguousarray(lower, np.float64)
        self.interfaces = list(interfaces) if interfaces else []
        if self._diag.shape[0] != addressing.size():
            raise ValueError("diag size differs from the number of cells")
        if self._upper.shape[0] != addressing.lowerAddr().shape[0]:
            raise ValueError("upper size differs from the number of faces")

    def lduAddr(self):
        return self._addr

    def diag(self):
        return self._diag

    def upper(self):
        return self._upper

    def lower(self):
        return self._upper if self._lower is None else self._lower

    def hasLower(self):
        return self._lower is not None

    def symmetric(self):
        return self._lower is None

    def asymmetric(self):
        return self._lower is not None


@dataclass
class solverPerformance:
    """SolverPerformance<scalar> plus the driver's profile/verbose figures."""

    solverName: str
    fieldName: str
    initialResidual: float = 0.0
    finalResidual: float = 0.0
    nIterations: int = 0
    converged: bool = False
    singular: bool = False
    nRestarts: int = 0
    deflated: bool = False
    polished: bool = False
    stagnated: bool = False
    normFactor: float = 0.0
    chebBeta: float = 0.0
    residualL2: float = 0.0
    timings: Dict[str, float] = field(default_factory=dict)

    def __str__(self):
        return (f"{self.solverName}:  Solving for {self.fieldName}, Initial residual = "
                f"{self.initialResidual:g}, Final residual = {self.finalResidual:g}, "
                f"No Iterations {self.nIterations}")


# One backend per (mesh, field): metalFoamSolver::backend() caches it in a
# static map keyed "field@meshptr" (metalFoamSolver.C:57-74).
_BACKENDS: Dict[tuple, "_lib.Context"] = {}


def backend_cache_clear():
    for ctx in _BACKENDS.values():
        ctx.close()
    _BACKENDS.clear()
    _TUNED.clear()


_CONTROL_KEYS = ("maxRestarts", "iterationsPerSync", "deflate", "chebyshevOrder",
                 "chebyshevRatio", "profile", "verbose", "graph", "stagnationLimit", "autotune",
                 "persistentMaxCells", "clusterMaxCells", "preconditioner", "nSweeps",
                 "nCellsInCoarsestLevel", "scaleCorrection", "smootherRatio")

def _preconditioner(name) -> int:
    """`preconditioner` of the cuda sub-dictionary: Chebyshev (the
    reference's Chebyshev-Jacobi, default) or GAMG (aggregation multigrid
    V-cycle, cudaPCG only)."""
    try:
        return _lib.PRECONDITIONERS[str(name)]
    except KeyError:
        raise FatalError(f"unknown preconditioner {name!r} in the cuda sub-dictionary "
                         f"(offered: {sorted(_lib.PRECONDITIONERS)})") from None


# backends whose SpMV launch shape has been chosen (autotune yes)
_TUNED: Dict[tuple, dict] = {}


class cudaFoamSolver:
    """Common FP64 driver of cudaPCG / cudaPBiCGStab (metalFoamSolver.H:60-108).

    ``controls`` is the fvSolution solver dictionary: ``tolerance``,
    ``relTol``, ``maxIter``, ``minIter`` and the optional sub-dictionary
    ``cuda`` (``metal`` is accepted too, so existing dictionaries work)
    with ``maxRestarts``, ``iterationsPerSync``, ``deflate``,
    ``chebyshevOrder``, ``chebyshevRatio``, ``profile``, ``verbose``,
    ``graph``, ``stagnationLimit``, ``autotune`` (pick the SpMV launch
    shape by timing, once per mesh and device, cached on disk; see
    :mod:`metal4foam_b200.autotune`), ``persistentMaxCells``,
    ``clusterMaxCells`` and, for cudaPCG, ``preconditioner`` (Chebyshev,
    the reference's default, or GAMG: one aggregation multigrid V-cycle per
    inner iteration) with ``nSweeps``, ``nCellsInCoarsestLevel``,
    ``scaleCorrection`` and ``smootherRatio``.
    """

    typeName = "cudaFoamSolver"
    useBiCGStab = False

    def __init__(self, fieldName: str, matrix: lduMatrix, controls: Optional[dict] = None,
                 interfaces=None, device: int = 0):
        self.fieldName_ = fieldName
        self.matrix_ = matrix
        self.controls_ = dict(controls or {})
        self.interfaces_ = list(interfaces) if interfaces is not None else list(matrix.interfaces)
        self.device_ = device
        sub = self.controls_.get("cuda", self.controls_.get("metal", {})) or {}
        unknown = set(sub) - set(_CONTROL_KEYS)
        if unknown:
            raise FatalError(f"unknown keys in the cuda sub-dictionary: {sorted(unknown)}")
        self.subDict_ = sub

    # metalFoamSolver::backend()
    def backend(self) -> "_lib.Context":
        key = (self.fieldName_, id(self.matrix_.lduAddr()), self.device_)
        ctx = _BACKENDS.get(key)
        if ctx is None:
            ctx = _lib.Context(self.device_)
            _BACKENDS[key] = ctx
            if self.subDict_.get("verbose", False):
                print("    " + ctx.description)
        return ctx

    def options(self):
        c = self.controls_
        s = self.subDict_
        return _lib.default_options(
            tolerance=float(c.get("tolerance", 1e-6)),
            relTol=float(c.get("relTol", 0.0)),
            maxIter=int(c.get("maxIter", 1000)),
            minIter=int(c.get("minIter", 0)),
            maxRestarts=int(s.get("maxRestarts", 8)),
            iterationsPerSync=int(s.get("iterationsPerSync", 1)),
            deflate=str(s.get("deflate", "auto")),
            chebyshevOrder=int(s.get("chebyshevOrder", 8)),
            chebyshevRatio=float(s.get("chebyshevRatio", 30.0)),
            profile=bool(s.get("profile", False)),
            verbose=bool(s.get("verbose", False)),
            graph=bool(s.get("graph", True)),
            stagnationLimit=int(s.get("stagnationLimit", 0)),
            persistentMaxCells=int(s.get("persistentMaxCells", 0)),
            clusterMaxCells=int(s.get("clusterMaxCells", 0)),
            preconditioner=_preconditioner(s.get("preconditioner", "Chebyshev")),
            nSweeps=int(s.get("nSweeps", 3)),
            nCellsInCoarsestLevel=int(s.get("nCellsInCoarsestLevel", 128)),
            scaleCorrection=float(s.get("scaleCorrection", 1.8)),
            smootherRatio=float(s.get("smootherRatio", 8.0)),
        )

    def solveImpl(self, psi: np.ndarray, source: np.ndarray, cmpt: int = 0) -> solverPerformance:
        # coupled interfaces are rejected (metalFoamSolver.C:89-99)
        if any(i is not None for i in self.interfaces_):
            raise FatalError(f"{self.typeName} does not support coupled boundaries "
                             "(processor/cyclic/AMI); run serially on a mesh without coupled "
                             "patches.")
        if not isinstance(psi, np.ndarray) or psi.dtype != np.float64 or not psi.flags["C_CONTIGUOUS"]:
            raise TypeError("psi must be a C-contiguous float64 array (updated in place)")
        src = np.ascontiguousarray(source, np.float64)
        m = self.matrix_
        a = m.lduAddr()
        bk = self.backend()
        if not bk.good:
            raise FatalError("CUDA backend unavailable: " + bk.description)
        bk.set_topology(a.size(), a.lowerAddr().shape[0], a.lowerAddr(), a.upperAddr(),
                        a.ownerStartAddr(), a.losortAddr(), a.losortStartAddr())
        tconv = bk.set_coeffs(m.diag(), m.upper(), m._lower)
        if self.subDict_.get("autotune", False):
            key = (self.fieldName_, id(a), self.device_)
            if key not in _TUNED:
                from types import SimpleNamespace

                from . import autotune
                shape = SimpleNamespace(n=a.size(), nf=a.lowerAddr().shape[0],
                                        lowerAddr=a.lowerAddr(), upperAddr=a.upperAddr())
                _TUNED[key] = autotune.tuned_config(bk, shape)
                if self.subDict_.get("verbose", False):
                    print(f"    {self.typeName}: SpMV launch shape {_TUNED[key]}")
        solver = _lib.CF_SOLVER_PBICGSTAB if self.useBiCGStab else _lib.CF_SOLVER_PCG
        p = bk.solve(solver, psi, src, self.options())
        return solverPerformance(
            solverName=self.typeName, fieldName=self.fieldName_,
            initialResidual=p.initialResidual, finalResidual=p.finalResidual,
            nIterations=p.nIterations, converged=bool(p.converged), singular=bool(p.singular),
            nRestarts=p.nRestarts, deflated=bool(p.deflated), polished=bool(p.polished),
            stagnated=bool(p.stagnated), normFactor=p.normFactor, chebBeta=p.chebBeta,
            residualL2=p.residualL2,
            timings=dict(tConvert=tconv + p.tConvert, tInner=p.tInner, tGpu=p.tGpu,
                         tSolve=p.tSolve))

    def solve(self, psi, source, cmpt: int = 0) -> solverPerformance:
        return self.solveImpl(psi, source, cmpt)

    def solveSegregated(self, psi: np.ndarray, source: np.ndarray):
        """All components of a vector equation on this matrix at once
        (fvMatrix<vector>::solveSegregated calls the scalar solver per
        component; here every SpMV serves all components): psi and source
        are C-contiguous float64 (nComponents, nCells), psi updated in place.
        Returns one solverPerformance per component, each equal to what
        solve() returns for that component alone.  cudaPBiCGStab only."""
        if not self.useBiCGStab:
            raise FatalError(f"{self.typeName}: segregated multi-component solves are "
                             "cudaPBiCGStab (momentum)")
        if any(i is not None for i in self.interfaces_):
            raise FatalError(f"{self.typeName} does not support coupled boundaries "
                             "(processor/cyclic/AMI); run serially on a mesh without coupled "
                             "patches.")
        if (not isinstance(psi, np.ndarray) or psi.dtype != np.float64 or psi.ndim != 2
                or not psi.flags["C_CONTIGUOUS"]):
            raise TypeError("psi must be a C-contiguous float64 (nComponents, nCells) array")
        src = np.ascontiguousarray(source, np.float64)
        if src.shape != psi.shape:
            raise ValueError("psi and source shapes differ")
        m = self.matrix_
        a = m.lduAddr()
        bk = self.backend()
        bk.set_topology(a.size(), a.lowerAddr().shape[0], a.lowerAddr(), a.upperAddr(),
                        a.ownerStartAddr(), a.losortAddr(), a.losortStartAddr())
        bk.set_coeffs(m.diag(), m.upper(), m._lower)
        out = []
        for k, p in enumerate(bk.solve_multi(_lib.CF_SOLVER_PBICGSTAB, psi, src, self.options())):
            out.append(solverPerformance(
                solverName=self.typeName, fieldName=f"{self.fieldName_}.component({k})",
                initialResidual=p.initialResidual, finalResidual=p.finalResidual,
                nIterations=p.nIterations, converged=bool(p.converged),
                singular=bool(p.singular), nRestarts=p.nRestarts, stagnated=bool(p.stagnated),
                normFactor=p.normFactor, residualL2=p.residualL2,
                timings=dict(tSolve=p.tSolve)))
        return out

    def scalarSolve(self, psi, source, cmpt: int = 0) -> solverPerformance:
        return self.solveImpl(psi, source, cmpt)


class cudaPCG(cudaFoamSolver):
    """Chebyshev-Jacobi PCG, FP32 inner on the GPU, FP64 refinement and
    constant-mode deflation on the GPU (metalPCG.H:47-92)."""

    typeName = "cudaPCG"
    useBiCGStab = False


class cudaPBiCGStab(cudaFoamSolver):
    """Jacobi BiCGStab, FP32 inner on the GPU, FP64 refinement on the GPU
    (metalPBiCGStab.H)."""

    typeName = "cudaPBiCGStab"
    useBiCGStab = True


# Run-time selection tables (addsymMatrixConstructorToTable /
# addasymMatrixConstructorToTable, metalPCG.C:18-19, metalPBiCGStab.C:18-22).
_SYM_TABLE = {"cudaPCG": cudaPCG, "cudaPBiCGStab": cudaPBiCGStab}
_ASYM_TABLE = {"cudaPBiCGStab": cudaPBiCGStab}


class _SolverSelector:
    @staticmethod
    def New(fieldName: str, matrix: lduMatrix, controls: dict, interfaces=None, device: int = 0):
        name = controls.get("solver")
        table = _SYM_TABLE if matrix.symmetric() else _ASYM_TABLE
        kind = "symmetric" if matrix.symmetric() else "asymmetric"
        if name not in table:
            raise FatalError(f"Unknown {kind} matrix solver {name}; valid solvers are "
                             f"{sorted(table)}")
        return table[name](fieldName, matrix, controls, interfaces, device)


lduMatrix.solver = _SolverSelector
