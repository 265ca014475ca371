"""ctypes binding of ``libcudafoam.so`` (the C ABI in include/cudafoam.h).

The library is the only compute path: if it is missing or no sm_100 device
is present, every call raises -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcudafoam.so")

CF_OK = 0
STATUS = {
    0: "CF_OK", 1: "CF_ERR_INVALID_ARG", 2: "CF_ERR_BAD_ADDRESSING", 3: "CF_ERR_NO_TOPOLOGY",
    4: "CF_ERR_NO_COEFFS", 5: "CF_ERR_CUDA", 6: "CF_ERR_NO_DEVICE", 7: "CF_ERR_DEVICE_TIMEOUT",
    8: "CF_ERR_UNSUPPORTED", 9: "CF_ERR_TOO_LARGE",
}
CF_SOLVER_PCG = 0
CF_SOLVER_PBICGSTAB = 1
DEFLATE = {"auto": 0, "on": 1, "off": 2}
CF_PRECOND_CHEBYSHEV = 0
CF_PRECOND_GAMG = 1
PRECONDITIONERS = {"Chebyshev": CF_PRECOND_CHEBYSHEV, "GAMG": CF_PRECOND_GAMG}
REORDER = {"none": 0, "rcm": 1, "auto": 2}


class CudaFoamError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class InnerStats(C.Structure):
    _fields_ = [
        ("nIterations", C.c_int32), ("converged", C.c_int32), ("singular", C.c_int32),
        ("stagnated", C.c_int32), ("finalResSum", C.c_double), ("tGpuSeconds", C.c_double),
        ("tWallSeconds", C.c_double),
    ]


class Options(C.Structure):
    _fields_ = [
        ("tolerance", C.c_double), ("relTol", C.c_double), ("maxIter", C.c_int32),
        ("minIter", C.c_int32), ("maxRestarts", C.c_int32), ("iterationsPerSync", C.c_int32),
        ("deflate", C.c_int32), ("chebyshevOrder", C.c_int32), ("chebyshevRatio", C.c_double),
        ("profile", C.c_int32), ("verbose", C.c_int32), ("graph", C.c_int32),
        ("stagnationLimit", C.c_int32),
        ("persistentMaxCells", C.c_int32),
        ("clusterMaxCells", C.c_int32),
        ("preconditioner", C.c_int32), ("nSweeps", C.c_int32),
        ("nCellsInCoarsestLevel", C.c_int32), ("scaleCorrection", C.c_double),
        ("smootherRatio", C.c_double),
    ]


class Performance(C.Structure):
    _fields_ = [
        ("initialResidual", C.c_double), ("finalResidual", C.c_double),
        ("nIterations", C.c_int32), ("nRestarts", C.c_int32), ("converged", C.c_int32),
        ("singular", C.c_int32), ("stagnated", C.c_int32), ("deflated", C.c_int32),
        ("polished", C.c_int32), ("solved", C.c_int32), ("normFactor", C.c_double),
        ("chebBeta", C.c_double), ("finalResSum32", C.c_double), ("residualL2", C.c_double),
        ("tConvert", C.c_double), ("tInner", C.c_double), ("tGpu", C.c_double),
        ("tSolve", C.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None

vp = C.c_void_p
i32 = C.c_int32
dbl = C.c_double

# (name, restype, argtypes) of every exported function
class SpmvConfig(C.Structure):
    _fields_ = [("layout", C.c_int32), ("rowsPerWarp", C.c_int32), ("blockSize", C.c_int32),
                ("rhsTile", C.c_int32), ("indexBits", C.c_int32)]

    def as_dict(self):
        return {"layout": LAYOUT_NAMES[self.layout], "rowsPerWarp": self.rowsPerWarp,
                "blockSize": self.blockSize, "rhsTile": self.rhsTile,
                "indexBits": self.indexBits}


class TuneEntry(C.Structure):
    _fields_ = [("config", SpmvConfig), ("msPerLaunch", C.c_double)]


class StepIO(C.Structure):
    """cf_step_io: vectors of one fused inner-iteration kernel (cf_inner_step)."""
    VECTORS = ["rA", "rA0", "wA", "pOld", "AyAOld", "delta", "zIn", "wIn", "p", "q", "yA",
               "AyA", "sA", "zA", "tA", "deltaNext", "rAOut", "wAOut", "wOut", "zOut"]
    _fields_ = ([(k, vp) for k in VECTORS] +
                [("alpha", C.c_double), ("beta", C.c_double), ("omega", C.c_double),
                 ("chebOrder", C.c_int32), ("chebStep", C.c_int32), ("chebBeta", C.c_double),
                 ("chebRatio", C.c_double), ("sums", C.c_double * 3)])


STEPS = {"cheb": 0, "pcg_p_spmv": 1, "pcg_update": 2, "bicg_ab": 3, "bicg_cd": 4, "bicg_e": 5}
# vectors each step writes (the others it reads)
STEP_OUTPUTS = {"cheb": ["wOut", "zOut"], "pcg_p_spmv": ["p", "q"],
                "pcg_update": ["deltaNext", "rAOut", "wAOut"],
                "bicg_ab": ["p", "yA", "AyA"], "bicg_cd": ["sA", "zA", "tA"],
                "bicg_e": ["deltaNext", "rAOut"]}

ALLREDUCE_FN = C.CFUNCTYPE(C.c_int, vp, vp, C.c_int32, C.c_int32, vp)
EXCHANGE_FN = C.CFUNCTYPE(C.c_int, vp, C.c_int32, vp, vp, C.c_int32, vp, vp, vp)
ABORT_FN = C.CFUNCTYPE(None, vp)


class Comm(C.Structure):
    """cf_comm: the subdomains' communication callbacks."""
    _fields_ = [("user", vp), ("allreduce", ALLREDUCE_FN), ("exchange", EXCHANGE_FN),
                ("abort", ABORT_FN), ("hostBuffers", C.c_int32)]


CF_LAYOUT_SELL32 = 0
CF_LAYOUT_LDU = 1
LAYOUTS = {"sell32": CF_LAYOUT_SELL32, "ldu": CF_LAYOUT_LDU}
LAYOUT_NAMES = {v: k for k, v in LAYOUTS.items()}


def spmv_config(layout="sell32", rowsPerWarp=32, blockSize=256, rhsTile=0, indexBits=16):
    return SpmvConfig(LAYOUTS[layout] if isinstance(layout, str) else int(layout),
                      int(rowsPerWarp), int(blockSize), int(rhsTile), int(indexBits))


SIGNATURES = [
    ("cf_abi_version", C.c_int, []),
    ("cf_last_error", C.c_char_p, []),
    ("cf_options_default", None, [C.POINTER(Options)]),
    ("cf_context_create", C.c_int, [C.POINTER(vp), i32]),
    ("cf_context_destroy", C.c_int, [vp]),
    ("cf_context_good", C.c_int, [vp]),
    ("cf_context_description", C.c_char_p, [vp]),
    ("cf_context_set_stream", C.c_int, [vp, vp]),
    ("cf_context_set_reorder", C.c_int, [vp, i32]),
    ("cf_context_kernel_launches", C.c_int, [vp, C.POINTER(C.c_longlong)]),
    ("cf_context_set_wait_limit", C.c_int, [vp, C.c_int64]),
    ("cf_set_topology", C.c_int, [vp, i32, i32, vp, vp, vp, vp, vp]),
    ("cf_set_coeffs", C.c_int, [vp, vp, vp, vp, C.POINTER(dbl)]),
    ("cf_set_coeffs_device", C.c_int, [vp, vp, vp, vp]),
    ("cf_pcg", C.c_int, [vp, vp, dbl, i32, i32, i32, dbl, dbl, C.POINTER(InnerStats)]),
    ("cf_bicgstab", C.c_int, [vp, vp, dbl, i32, C.POINTER(InnerStats)]),
    ("cf_delta", C.c_int, [vp, vp]),
    ("cf_solve", C.c_int, [vp, i32, vp, vp, C.POINTER(Options), C.POINTER(Performance)]),
    ("cf_solve_device", C.c_int, [vp, i32, vp, vp, C.POINTER(Options), C.POINTER(Performance)]),
    ("cf_residual", C.c_int, [vp, i32, vp]),
    ("cf_spmv_config_default", C.c_int, [C.POINTER(SpmvConfig)]),
    ("cf_get_spmv_config", C.c_int, [vp, C.POINTER(SpmvConfig)]),
    ("cf_set_spmv_config", C.c_int, [vp, C.POINTER(SpmvConfig)]),
    ("cf_autotune", C.c_int, [vp, i32, i32, C.POINTER(SpmvConfig), C.POINTER(TuneEntry), i32,
                              C.POINTER(i32)]),
    ("cf_gamg_levels", C.c_int, [vp, C.POINTER(i32), i32, C.POINTER(i32)]),
    ("cf_solve_many_device", C.c_int, [C.POINTER(vp), i32, i32, C.POINTER(vp), C.POINTER(vp),
                                       C.POINTER(vp), C.POINTER(vp), C.POINTER(vp),
                                       C.POINTER(Options), i32, vp]),
    ("cf_gamg_export", C.c_int, [vp, i32, C.POINTER(i32), vp, vp, vp, vp, vp]),
    ("cf_solve_multi", C.c_int, [vp, i32, i32, vp, vp, C.POINTER(Options),
                                 C.POINTER(Performance)]),
    ("cf_solve_multi_device", C.c_int, [vp, i32, i32, vp, vp, C.POINTER(Options),
                                        C.POINTER(Performance)]),
    ("cf_batch_create", C.c_int, [C.POINTER(vp), i32]),
    ("cf_batch_destroy", C.c_int, [vp]),
    ("cf_batch_set_stream", C.c_int, [vp, vp]),
    ("cf_batch_kernel_launches", C.c_int, [vp, C.POINTER(C.c_longlong)]),
    ("cf_batch_add_system", C.c_int, [vp, i32, i32, vp, vp, vp, vp, vp, C.POINTER(i32)]),
    ("cf_batch_finalize", C.c_int, [vp, i32]),
    ("cf_batch_set_solo_cells", C.c_int, [vp, i32]),
    ("cf_batch_set_coeffs", C.c_int, [vp, i32, vp, vp, vp]),
    ("cf_batch_set_coeffs_device", C.c_int, [vp, i32, vp, vp, vp]),
    ("cf_batch_solve", C.c_int, [vp, i32, C.POINTER(vp), C.POINTER(vp), C.POINTER(Options),
                                 C.POINTER(Performance)]),
    ("cf_batch_solve_device", C.c_int, [vp, i32, C.POINTER(vp), C.POINTER(vp),
                                        C.POINTER(Options), C.POINTER(Performance)]),
    ("cf_set_transpose", C.c_int, [vp, i32]),
    ("cf_face_gradients", C.c_int, [vp, vp, vp, vp, vp, vp]),
    ("cf_face_gradients_device", C.c_int, [vp, vp, vp, vp, vp, vp]),
    ("cf_solve_adjoint", C.c_int, [vp, i32, vp, vp, vp, vp, vp, vp, C.POINTER(Options),
                                   C.POINTER(Performance)]),
    ("cf_solve_adjoint_device", C.c_int, [vp, i32, vp, vp, vp, vp, vp, vp, C.POINTER(Options),
                                          C.POINTER(Performance)]),
    ("cf_amul", C.c_int, [vp, vp, vp, i32]),
    ("cf_spmv32", C.c_int, [vp, vp, vp, vp, C.POINTER(dbl)]),
    ("cf_cheb_apply", C.c_int, [vp, vp, vp, i32, dbl, dbl]),
    ("cf_time_kernel", C.c_int, [vp, i32, i32, C.POINTER(dbl)]),
    ("cf_inner_step", C.c_int, [vp, i32, C.POINTER(StepIO)]),
    ("cf_subdomain_create", C.c_int, [C.POINTER(vp), i32]),
    ("cf_subdomain_destroy", C.c_int, [vp]),
    ("cf_subdomain_set_stream", C.c_int, [vp, vp]),
    ("cf_subdomain_kernel_launches", C.c_int, [vp, C.POINTER(C.c_longlong)]),
    ("cf_subdomain_set_topology", C.c_int, [vp, i32, i32, vp, vp, vp, vp, vp, i32, vp, vp, vp,
                                            i32]),
    ("cf_subdomain_set_coeffs", C.c_int, [vp, vp, vp, vp, vp]),
    ("cf_subdomain_solve", C.c_int, [vp, i32, vp, vp, C.POINTER(Options), C.POINTER(Comm),
                                     C.POINTER(Performance)]),
    ("cf_comm_local_create", C.c_int, [i32, C.c_double, C.POINTER(Comm)]),
    ("cf_comm_local_destroy", C.c_int, [i32, C.POINTER(Comm)]),
    ("cf_ldu_spmv_dot_noalloc", C.c_int, [i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp,
                                          vp]),
]


def load():
    """Load libcudafoam.so (building it first when absent and nvcc exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        from . import build as _build
        _build.build()
    if not os.path.exists(LIB_PATH):
        raise CudaFoamError(6, f"{LIB_PATH} is missing; run python -m metal4foam_b200.build")
    L = C.CDLL(LIB_PATH)
    for name, res, args in SIGNATURES:
        fn = getattr(L, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def check(rc):
    if rc != CF_OK:
        msg = load().cf_last_error()
        raise CudaFoamError(rc, msg.decode() if msg else "")
    return rc


def ptr(a):
    """Pointer of a C-contiguous numpy array, a torch tensor, or None."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("array must be C-contiguous")
        return a.ctypes.data_as(vp)
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return vp(a.data_ptr())
    raise TypeError(f"unsupported array type {type(a)}")


def solve_many_device(contexts, solver, psis, sources, options, streams=8, diags=None,
                      uppers=None, lowers=None):
    """cf_solve_many_device: independent systems (one Context each) solved
    concurrently on `streams` host threads / CUDA streams; device arrays
    (torch tensors); coefficients staged first when diags is given.
    Returns one Performance per system."""
    n = len(contexts)
    arr = vp * max(n, 1)
    ctx = arr(*[c.h for c in contexts])
    ps = arr(*[ptr(x) for x in psis])
    ss = arr(*[ptr(x) for x in sources])
    ds = arr(*[ptr(x) for x in diags]) if diags is not None else None
    us = arr(*[ptr(x) for x in uppers]) if uppers is not None else None
    ls = arr(*[ptr(x) for x in lowers]) if lowers is not None else None
    perf = (Performance * max(n, 1))()
    check(load().cf_solve_many_device(ctx, int(n), int(solver), ps, ss, ds, us, ls,
                                      C.byref(options), int(streams), perf))
    return list(perf)[:n]


def default_options(**kw):
    o = Options()
    load().cf_options_default(C.byref(o))
    for k, v in kw.items():
        if k == "deflate" and isinstance(v, str):
            v = DEFLATE[v]
        if k == "preconditioner" and isinstance(v, str):
            v = PRECONDITIONERS[v]
        if isinstance(v, bool):
            v = int(v)
        if not hasattr(o, k):
            raise KeyError(f"unknown option {k}")
        setattr(o, k, v)
    return o


class Context:
    """One device context = one (mesh, field) backend of the reference
    (metalFoamSolver::backend(), metalFoamSolver.C:57-74)."""

    def __init__(self, device: int = 0, reorder: str = "auto"):
        L = load()
        h = vp()
        check(L.cf_context_create(C.byref(h), int(device)))
        self.h = h
        self._keep = {}
        self.reorder = reorder
        check(L.cf_context_set_reorder(self.h, REORDER[reorder]))

    def close(self):
        if getattr(self, "h", None):
            load().cf_context_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def description(self) -> str:
        return load().cf_context_description(self.h).decode()

    @property
    def good(self) -> bool:
        return bool(load().cf_context_good(self.h))

    def kernel_launches(self) -> int:
        n = C.c_longlong()
        check(load().cf_context_kernel_launches(self.h, C.byref(n)))
        return n.value

    def set_wait_limit(self, polls=0):
        check(load().cf_context_set_wait_limit(self.h, int(polls)))

    def set_stream(self, stream_handle):
        check(load().cf_context_set_stream(self.h, vp(stream_handle) if stream_handle else None))

    def set_topology(self, n, nf, low, upp, own, los, losS):
        arrs = [np.ascontiguousarray(a, np.int32) for a in (low, upp, own, los, losS)]
        self._keep["topo"] = arrs   # the cache key is the pointer identity
        check(load().cf_set_topology(self.h, int(n), int(nf), *(ptr(a) for a in arrs)))

    def set_coeffs(self, diag, upper, lower=None):
        d = np.ascontiguousarray(diag, np.float64)
        u = np.ascontiguousarray(upper, np.float64)
        l = None if lower is None else np.ascontiguousarray(lower, np.float64)
        t = C.c_double()
        check(load().cf_set_coeffs(self.h, ptr(d), ptr(u), ptr(l), C.byref(t)))
        return t.value

    def set_coeffs_device(self, diag, upper, lower=None):
        check(load().cf_set_coeffs_device(self.h, ptr(diag), ptr(upper), ptr(lower)))

    def pcg(self, r, target, maxIter, iterationsPerSync=1, chebOrder=1, chebBeta=2.0,
            chebRatio=30.0):
        st = InnerStats()
        rr = np.ascontiguousarray(r, np.float64)
        check(load().cf_pcg(self.h, ptr(rr), float(target), int(maxIter),
                            int(iterationsPerSync), int(chebOrder), float(chebBeta),
                            float(chebRatio), C.byref(st)))
        return st

    def bicgstab(self, r, target, maxIter):
        st = InnerStats()
        rr = np.ascontiguousarray(r, np.float64)
        check(load().cf_bicgstab(self.h, ptr(rr), float(target), int(maxIter), C.byref(st)))
        return st

    def delta(self, n):
        out = np.empty(n, np.float32)
        check(load().cf_delta(self.h, ptr(out)))
        return out

    def solve(self, solver, psi, source, options):
        perf = Performance()
        check(load().cf_solve(self.h, int(solver), ptr(psi), ptr(source), C.byref(options),
                              C.byref(perf)))
        return perf

    def solve_device(self, solver, psi, source, options):
        perf = Performance()
        check(load().cf_solve_device(self.h, int(solver), ptr(psi), ptr(source),
                                     C.byref(options), C.byref(perf)))
        return perf

    def solve_multi(self, solver, psi, source, options):
        """psi, source: C-contiguous float64 (nrhs, nCells); psi in place."""
        nrhs = int(psi.shape[0])
        if source.shape != psi.shape:
            raise ValueError("psi and source shapes differ")
        perf = (Performance * nrhs)()
        check(load().cf_solve_multi(self.h, int(solver), nrhs, ptr(psi), ptr(source),
                                    C.byref(options), perf))
        return list(perf)

    def solve_multi_device(self, solver, psi, source, options):
        """psi, source: device tensors (nrhs, nCells) float64."""
        nrhs = int(psi.shape[0])
        perf = (Performance * nrhs)()
        check(load().cf_solve_multi_device(self.h, int(solver), nrhs, ptr(psi), ptr(source),
                                           C.byref(options), perf))
        return list(perf)

    def set_transpose(self, on=True):
        check(load().cf_set_transpose(self.h, int(bool(on))))

    def face_gradients(self, lam, x, nf):
        lam = np.ascontiguousarray(lam, np.float64)
        x = np.ascontiguousarray(x, np.float64)
        dU = np.empty(nf)
        dL = np.empty(nf)
        dD = np.empty_like(x)
        check(load().cf_face_gradients(self.h, ptr(lam), ptr(x), ptr(dU), ptr(dL), ptr(dD)))
        return dU, dL, dD

    def solve_adjoint(self, solver, x, dLdx, nf, options):
        x = np.ascontiguousarray(x, np.float64)
        g = np.ascontiguousarray(dLdx, np.float64)
        lam = np.empty_like(x)
        dU = np.empty(nf)
        dL = np.empty(nf)
        dD = np.empty_like(x)
        perf = Performance()
        check(load().cf_solve_adjoint(self.h, int(solver), ptr(x), ptr(g), ptr(lam), ptr(dU),
                                      ptr(dL), ptr(dD), C.byref(options), C.byref(perf)))
        return lam, dU, dL, dD, perf

    def residual(self, n, which="final"):
        out = np.empty(n)
        check(load().cf_residual(self.h, {"initial": 0, "final": 1}[which], ptr(out)))
        return out

    def amul(self, x, transpose=False):
        xx = np.ascontiguousarray(x, np.float64)
        y = np.empty_like(xx)
        check(load().cf_amul(self.h, ptr(xx), ptr(y), int(transpose)))
        return y

    def spmv32(self, x, w=None):
        xx = np.ascontiguousarray(x, np.float32)
        ww = None if w is None else np.ascontiguousarray(w, np.float32)
        y = np.empty_like(xx)
        d = C.c_double()
        check(load().cf_spmv32(self.h, ptr(xx), ptr(ww), ptr(y), C.byref(d)))
        return y, d.value

    KERNELS = {"cheb_step": 0, "spmv32": 1, "pcg_p_spmv": 2, "pcg_update": 3, "amul64": 4,
               "cheb_step_inner": 5, "spmv32_cold": 6}

    def time_kernel(self, which, reps=50):
        ms = C.c_double()
        check(load().cf_time_kernel(self.h, self.KERNELS[which], int(reps), C.byref(ms)))
        return ms.value

    def spmv_config(self):
        k = SpmvConfig()
        check(load().cf_get_spmv_config(self.h, C.byref(k)))
        return k

    def set_spmv_config(self, cfg=None, **kw):
        """Launch shape of the FP32 SpMV kernels: pass a SpmvConfig, or
        keywords of :func:`spmv_config` (unnamed ones keep their defaults)."""
        k = cfg if cfg is not None else spmv_config(**kw)
        check(load().cf_set_spmv_config(self.h, C.byref(k)))

    def gamg_levels(self):
        """Cells per level of the GAMG hierarchy ([] before any GAMG solve)."""
        cells = (C.c_int32 * 32)()
        nl = C.c_int32()
        check(load().cf_gamg_levels(self.h, cells, 32, C.byref(nl)))
        return [cells[i] for i in range(min(nl.value, 32))]

    def gamg_export(self, level):
        """Level `level` (>= 1) of the GAMG hierarchy: (agg of the finer
        level's cells, diag, upper, lowerAddr, upperAddr)."""
        cells = self.gamg_levels()
        nf = C.c_int32()
        check(load().cf_gamg_export(self.h, int(level), C.byref(nf), None, None, None, None,
                                    None))
        agg = np.empty(cells[level - 1], np.int32)
        diag = np.empty(cells[level], np.float64)
        upper = np.empty(nf.value, np.float64)
        lo = np.empty(nf.value, np.int32)
        up = np.empty(nf.value, np.int32)
        check(load().cf_gamg_export(self.h, int(level), C.byref(nf), ptr(agg), ptr(diag),
                                    ptr(upper), ptr(lo), ptr(up)))
        return agg, diag, upper, lo, up

    def autotune(self, reps=20, apply=True):
        """Times every SpMV launch shape on this matrix; returns (best
        config, [(config dict, ms per launch), ...])."""
        best = SpmvConfig()
        table = (TuneEntry * 64)()
        count = C.c_int32()
        check(load().cf_autotune(self.h, int(reps), int(bool(apply)), C.byref(best), table, 64,
                                 C.byref(count)))
        return best, [(table[i].config.as_dict(), table[i].msPerLaunch)
                      for i in range(min(count.value, 64))]

    def inner_step(self, step, n, alpha=0.0, beta=0.0, omega=0.0, chebOrder=1, chebStep=0,
                   chebBeta=2.0, chebRatio=30.0, **vectors):
        """One launch of a fused inner-iteration kernel (cf_inner_step):
        `vectors` are the step's FP32 inputs by name; returns (outputs by
        name, sums)."""
        io = StepIO()
        keep = []
        for k, v in vectors.items():
            a = np.ascontiguousarray(v, np.float32)
            keep.append(a)
            setattr(io, k, a.ctypes.data)
        outs = {}
        for k in STEP_OUTPUTS[step]:
            if k in vectors:     # an input the step also writes is not an output slot
                continue
            outs[k] = np.empty(n, np.float32)
            setattr(io, k, outs[k].ctypes.data)
        io.alpha, io.beta, io.omega = float(alpha), float(beta), float(omega)
        io.chebOrder, io.chebStep = int(chebOrder), int(chebStep)
        io.chebBeta, io.chebRatio = float(chebBeta), float(chebRatio)
        check(load().cf_inner_step(self.h, STEPS[step], C.byref(io)))
        return outs, list(io.sums)

    def cheb_apply(self, r, order, beta, ratio=30.0):
        rr = np.ascontiguousarray(r, np.float32)
        z = np.empty_like(rr)
        check(load().cf_cheb_apply(self.h, ptr(rr), ptr(z), int(order), float(beta),
                                   float(ratio)))
        return z


class Batch:
    """Many independent symmetric systems solved together (cf_batch_*)."""

    def __init__(self, device: int = 0):
        h = vp()
        check(load().cf_batch_create(C.byref(h), int(device)))
        self.h = h
        self.sizes = []

    def close(self):
        if getattr(self, "h", None):
            load().cf_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_system(self, addr):
        arrs = [np.ascontiguousarray(a, np.int32) for a in addr.arrays()]
        idx = C.c_int32()
        check(load().cf_batch_add_system(self.h, int(addr.n), int(addr.nf),
                                         *(ptr(a) for a in arrs), C.byref(idx)))
        self.sizes.append((addr.n, addr.nf))
        return idx.value

    def set_solo_cells(self, min_cells):
        check(load().cf_batch_set_solo_cells(self.h, int(min_cells)))

    def finalize(self, reorder="auto"):
        check(load().cf_batch_finalize(self.h, REORDER[reorder]))

    def set_stream(self, stream_handle):
        check(load().cf_batch_set_stream(self.h, vp(stream_handle) if stream_handle else None))

    def kernel_launches(self):
        n = C.c_longlong()
        check(load().cf_batch_kernel_launches(self.h, C.byref(n)))
        return n.value

    def set_coeffs(self, i, diag, upper):
        d = np.ascontiguousarray(diag, np.float64)
        u = np.ascontiguousarray(upper, np.float64)
        check(load().cf_batch_set_coeffs(self.h, int(i), ptr(d), ptr(u), None))

    def set_coeffs_device(self, i, diag, upper):
        check(load().cf_batch_set_coeffs_device(self.h, int(i), ptr(diag), ptr(upper), None))

    def _solve(self, fn, psis, sources, options):
        S = len(self.sizes)
        pp = (vp * S)(*[ptr(p).value if ptr(p) is not None else None for p in psis])
        ss = (vp * S)(*[ptr(s).value if ptr(s) is not None else None for s in sources])
        perf = (Performance * S)()
        check(fn(self.h, CF_SOLVER_PCG, pp, ss, C.byref(options), perf))
        return list(perf)

    def solve(self, psis, sources, options):
        """psis: list of float64 arrays (updated in place), sources: list."""
        srcs = [np.ascontiguousarray(s, np.float64) for s in sources]
        return self._solve(load().cf_batch_solve, psis, srcs, options)

    def solve_device(self, psis, sources, options):
        return self._solve(load().cf_batch_solve_device, psis, sources, options)


class SubdomainSolver:
    """One subdomain of a decomposed system (cf_subdomain_*): its internal
    LDU matrix plus processor interfaces (metal4foam_b200.decompose)."""

    def __init__(self, sub, device: int = 0, reorder: str = "auto"):
        L = load()
        h = vp()
        check(L.cf_subdomain_create(C.byref(h), int(device)))
        self.h = h
        self.sub = sub
        s = sub.system
        a = s.addr
        nb, nfc, fc, cf = sub.interface_arrays()
        self._keep = (a.arrays(), nb, nfc, fc)
        check(L.cf_subdomain_set_topology(self.h, a.n, a.nf, *(ptr(x) for x in a.arrays()),
                                          len(nb), ptr(nb), ptr(nfc), ptr(fc), REORDER[reorder]))
        self.set_coeffs(s.diag, s.upper, s.lower, cf)

    def set_coeffs(self, diag, upper, lower, interfaceCoeffs):
        d = np.ascontiguousarray(diag, np.float64)
        u = np.ascontiguousarray(upper, np.float64)
        lo = None if lower is None else np.ascontiguousarray(lower, np.float64)
        c = np.ascontiguousarray(interfaceCoeffs, np.float64)
        check(load().cf_subdomain_set_coeffs(self.h, ptr(d), ptr(u), ptr(lo), ptr(c)))

    def set_stream(self, stream_handle):
        check(load().cf_subdomain_set_stream(self.h, vp(stream_handle) if stream_handle else None))

    def solve(self, solver, psi, source, options, comm):
        """psi (float64, this subdomain's cells) is updated in place; comm is
        a Comm structure; returns the Performance (raises on failure)."""
        assert psi.dtype == np.float64 and psi.flags.c_contiguous
        src = np.ascontiguousarray(source, np.float64)
        perf = Performance()
        rc = load().cf_subdomain_solve(self.h, int(solver), ptr(psi), ptr(src),
                                       C.byref(options), C.byref(comm), C.byref(perf))
        check(rc)
        return perf

    def kernel_launches(self):
        n = C.c_longlong()
        check(load().cf_subdomain_kernel_launches(self.h, C.byref(n)))
        return n.value

    def close(self):
        if getattr(self, "h", None):
            load().cf_subdomain_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class LocalComm:
    """The in-process communicator of cf_comm_local_create: nRanks Comm
    structures for nRanks threads of this process."""

    def __init__(self, nRanks: int, timeoutSeconds: float = 120.0):
        self.n = int(nRanks)
        self.comms = (Comm * self.n)()
        check(load().cf_comm_local_create(self.n, float(timeoutSeconds), self.comms))

    def __getitem__(self, r):
        return self.comms[r]

    def close(self):
        if getattr(self, "comms", None) is not None:
            load().cf_comm_local_destroy(self.n, self.comms)
            self.comms = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
