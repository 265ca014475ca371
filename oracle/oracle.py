"""ctypes front end of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg import this module, and only as the checker / the timed CPU path; the
product (``metal4foam_b200``) never imports it.

``liboracle.so`` is the C restatement (oracle/*.c); ``libmslref.so`` is the
reference's own MSL kernel source compiled on the CPU through
``oracle/msl_shim`` (only present where the reference was available at
build time).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libmslref.so")

_lib = None
_ref = None

i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")


class Controls(C.Structure):
    _fields_ = [
        ("tolerance", C.c_double),
        ("relTol", C.c_double),
        ("maxIter", C.c_int32),
        ("minIter", C.c_int32),
        ("maxRestarts", C.c_int32),
        ("iterationsPerSync", C.c_int32),
        ("deflate", C.c_int32),
        ("chebyshevOrder", C.c_int32),
        ("chebyshevRatio", C.c_double),
    ]


class Perf(C.Structure):
    _fields_ = [
        ("initialResidual", C.c_double),
        ("finalResidual", C.c_double),
        ("nIterations", C.c_int32),
        ("nRestarts", C.c_int32),
        ("singular", C.c_int32),
        ("converged", C.c_int32),
        ("deflated", C.c_int32),
        ("polished", C.c_int32),
        ("solved", C.c_int32),
        ("chebBeta", C.c_double),
        ("normFactor", C.c_double),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("nIterations", C.c_int32),
        ("finalResSum", C.c_double),
        ("converged", C.c_int32),
        ("singular", C.c_int32),
        ("stagnated", C.c_int32),
    ]


class FoamPerf(C.Structure):
    _fields_ = [
        ("initialResidual", C.c_double),
        ("finalResidual", C.c_double),
        ("nIterations", C.c_int32),
        ("converged", C.c_int32),
        ("singular", C.c_int32),
    ]


class Ldu32(C.Structure):
    _fields_ = [
        ("n", C.c_int32), ("nf", C.c_int32),
        ("diag", C.c_void_p), ("upper", C.c_void_p), ("lower", C.c_void_p),
        ("low", C.c_void_p), ("upp", C.c_void_p), ("ownStart", C.c_void_p),
        ("losort", C.c_void_p), ("losortStart", C.c_void_p),
    ]


def build():
    """Compile liboracle.so (and libmslref.so when the reference is here)."""
    import subprocess
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    ref = reference_dir()
    if os.path.isdir(os.path.join(ref, "src")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REFERENCE_DIR={ref}"], check=True)


def reference_dir():
    """The reference checkout: $REFERENCE_DIR, else the directory
    `reference` beside this repository's root (absent on machines that only
    use the prebuilt oracle)."""
    return os.environ.get("REFERENCE_DIR") or os.path.normpath(
        os.path.join(HERE, "..", "..", "reference"))


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.orc_build_addressing.argtypes = [C.c_int32, C.c_int32, i32p, i32p, i32p, i32p, i32p]
        L.orc_build_addressing.restype = C.c_int
        for nm in ("orc_amul", "orc_tmul"):
            getattr(L, nm).argtypes = [C.c_int32, C.c_int32, i32p, i32p, f64p, f64p, C.c_void_p, f64p, f64p]
            getattr(L, nm).restype = None
        L.orc_sumA.argtypes = [C.c_int32, C.c_int32, i32p, i32p, f64p, f64p, C.c_void_p, f64p]
        L.orc_normfactor.argtypes = [C.c_int32, f64p, f64p, f64p, f64p]
        L.orc_normfactor.restype = C.c_double
        L.orc_sum_mag.argtypes = [C.c_int32, f64p]
        L.orc_sum_mag.restype = C.c_double
        L.orc_check_convergence.argtypes = [C.c_double] * 4
        L.orc_check_convergence.restype = C.c_int
        L.orc_metal_solve.argtypes = [C.c_int32, C.c_int32, i32p, i32p, i32p, i32p, i32p,
                                      f64p, f64p, C.c_void_p, f64p, f64p, C.c_int32,
                                      C.POINTER(Controls), C.POINTER(Perf)]
        L.orc_metal_solve.restype = C.c_int
        L.orc_foam_pcg.argtypes = [C.c_int32, C.c_int32, i32p, i32p, i32p, i32p, i32p,
                                   f64p, f64p, f64p, f64p, C.c_int32, C.c_double,
                                   C.c_double, C.c_int32, C.c_int32, C.c_int32,
                                   C.POINTER(FoamPerf)]
        L.orc_foam_pbicgstab.argtypes = [C.c_int32, C.c_int32, i32p, i32p, i32p, i32p, i32p,
                                         f64p, f64p, f64p, f64p, f64p, C.c_double,
                                         C.c_double, C.c_int32, C.c_int32, C.c_int32,
                                         C.POINTER(FoamPerf)]
        L.orc_cg64.argtypes = [C.c_int32, C.c_int32, i32p, i32p, i32p, i32p, i32p, f64p,
                               f64p, C.c_void_p, f64p, f64p, C.c_double, C.c_int32,
                               C.c_int32, C.c_int32]
        L.orc_cg64.restype = C.c_int
        L.orc_face_gradients.argtypes = [C.c_int32, C.c_int32, i32p, i32p, f64p, f64p,
                                         f64p, f64p, f64p]
        L.orc_amul_rows.argtypes = [C.c_int32, i32p, i32p, i32p, i32p, i32p, f64p, f64p,
                                    C.c_void_p, f64p, f64p, C.c_int32, C.c_int32]
        L.orc_backend_new.argtypes = [C.c_int32, C.c_int32, i32p, i32p, i32p, i32p, i32p]
        L.orc_backend_new.restype = C.c_void_p
        L.orc_backend_free.argtypes = [C.c_void_p]
        L.orc_backend_set_coeffs.argtypes = [C.c_void_p, f64p, f64p, C.c_void_p]
        L.orc_backend_pcg.argtypes = [C.c_void_p, f64p, C.c_double, C.c_int32, C.c_int32,
                                      C.c_int32, C.c_double, C.c_double]
        L.orc_backend_pcg.restype = Stats
        L.orc_backend_bicgstab.argtypes = [C.c_void_p, f64p, C.c_double, C.c_int32]
        L.orc_backend_bicgstab.restype = Stats
        L.orc_backend_delta.argtypes = [C.c_void_p]
        L.orc_backend_delta.restype = C.POINTER(C.c_float)
        L.orc_cheb_constants.argtypes = [C.c_int32, C.c_double, C.c_double, f32p]
        # kernels
        L.orc_k_ldu_spmv_dotw.argtypes = [C.POINTER(Ldu32), f32p, f32p, f32p, f32p]
        L.orc_k_ldu_spmv.argtypes = [C.POINTER(Ldu32), f32p, f32p]
        L.orc_k_cheb_init.argtypes = [C.c_int32, f32p, f32p, f32p, f32p, C.c_float]
        L.orc_k_cheb_step.argtypes = [C.c_int32, f32p, f32p, f32p, f32p, f32p, C.c_float, C.c_float]
        L.orc_k_emul.argtypes = [C.c_int32, f32p, f32p, f32p]
        L.orc_k_pcg_precond_dot.argtypes = [C.c_int32, f32p, f32p, f32p, f32p]
        L.orc_k_pcg_update_p.argtypes = [C.c_int32, f32p, f32p, f32p]
        L.orc_k_pcg_update_sol_res.argtypes = [C.c_int32, f32p, f32p, f32p, f32p, f32p, f32p]
        L.orc_k_dot_partial.argtypes = [C.c_int32, f32p, f32p, f32p]
        L.orc_k_reduce_scalars.argtypes = [f32p, f32p, f32p, C.c_uint32, C.c_uint32, C.c_uint32]
        L.orc_k_bicg_update_p.argtypes = [C.c_int32, f32p, f32p, f32p, f32p]
        L.orc_k_bicg_s_res.argtypes = [C.c_int32, f32p, f32p, f32p, f32p, f32p]
        L.orc_k_bicg_early_update.argtypes = [C.c_int32, f32p, f32p, f32p]
        L.orc_k_bicg_update_sol_res.argtypes = [C.c_int32, f32p, f32p, f32p, f32p, f32p, f32p, f32p, f32p]
        _lib = L
    return _lib


def ref_lib():
    """The reference's own kernels compiled for the CPU, or None."""
    global _ref
    if _ref is None and os.path.exists(REF_PATH):
        _ref = C.CDLL(REF_PATH)
    return _ref


def _addr(sysm):
    a = sysm.addr
    return (a.n, a.nf, a.lowerAddr, a.upperAddr, a.ownerStartAddr, a.losortAddr,
            a.losortStartAddr)


def _ptr_or_none(arr):
    return None if arr is None else arr.ctypes.data_as(C.c_void_p)


def build_addressing(n, low, upp):
    nf = len(low)
    own = np.zeros(n + 1, np.int32)
    lo = np.zeros(max(nf, 1), np.int32)
    los = np.zeros(n + 1, np.int32)
    rc = lib().orc_build_addressing(n, nf, np.ascontiguousarray(low, np.int32),
                                    np.ascontiguousarray(upp, np.int32), own, lo, los)
    if rc != 0:
        raise ValueError("faces not in LDU order")
    return own, lo[:nf], los


def amul(sysm, x, transpose=False):
    y = np.empty(sysm.n)
    fn = lib().orc_tmul if transpose else lib().orc_amul
    lower = sysm.lower
    fn(sysm.n, sysm.nf, sysm.addr.lowerAddr, sysm.addr.upperAddr, sysm.diag, sysm.upper,
       _ptr_or_none(lower), np.ascontiguousarray(x, np.float64), y)
    return y


def sumA(sysm):
    u = np.empty(sysm.n)
    lib().orc_sumA(sysm.n, sysm.nf, sysm.addr.lowerAddr, sysm.addr.upperAddr, sysm.diag,
                   sysm.upper, _ptr_or_none(sysm.lower), u)
    return u


def normfactor(psi, source, Apsi, sumA_):
    return lib().orc_normfactor(len(psi), *(np.ascontiguousarray(v, np.float64)
                                            for v in (psi, source, Apsi, sumA_)))


def check_convergence(tol, relTol, initial, final):
    return bool(lib().orc_check_convergence(tol, relTol, initial, final))


@dataclass
class SolveResult:
    psi: np.ndarray
    initialResidual: float
    finalResidual: float
    nIterations: int
    nRestarts: int
    singular: bool
    converged: bool
    deflated: bool
    polished: bool
    chebBeta: float
    normFactor: float


def controls(tolerance=1e-6, relTol=0.0, maxIter=1000, minIter=0, maxRestarts=8,
             iterationsPerSync=1, deflate="auto", chebyshevOrder=8, chebyshevRatio=30.0):
    d = {"auto": 0, "on": 1, "off": 2}[deflate] if isinstance(deflate, str) else int(deflate)
    return Controls(tolerance, relTol, maxIter, minIter, maxRestarts, iterationsPerSync, d,
                    chebyshevOrder, chebyshevRatio)


def metal_solve(sysm, bicgstab=False, psi=None, **kw):
    """The reference algorithm (FP32 inner emulation + FP64 driver)."""
    ctl = controls(**kw)
    psi = np.array(sysm.psi if psi is None else psi, dtype=np.float64, copy=True)
    perf = Perf()
    lib().orc_metal_solve(*_addr(sysm), sysm.diag, sysm.upper, _ptr_or_none(sysm.lower), psi,
                          np.ascontiguousarray(sysm.source, np.float64), int(bicgstab),
                          C.byref(ctl), C.byref(perf))
    return SolveResult(psi, perf.initialResidual, perf.finalResidual, perf.nIterations,
                       perf.nRestarts, bool(perf.singular), bool(perf.converged),
                       bool(perf.deflated), bool(perf.polished), perf.chebBeta, perf.normFactor)


PRECOND = {"none": 0, "diagonal": 1, "DIC": 2}


def foam_pcg(sysm, precond="DIC", tolerance=1e-6, relTol=0.0, maxIter=1000, minIter=0,
             nthreads=1, psi=None, source=None):
    psi = np.array(sysm.psi if psi is None else psi, dtype=np.float64, copy=True)
    src = np.ascontiguousarray(sysm.source if source is None else source, np.float64)
    perf = FoamPerf()
    lib().orc_foam_pcg(*_addr(sysm), sysm.diag, sysm.upper, psi, src, PRECOND[precond],
                       tolerance, relTol, maxIter, minIter, nthreads, C.byref(perf))
    return psi, perf


def foam_pbicgstab(sysm, tolerance=1e-6, relTol=0.0, maxIter=1000, minIter=0, nthreads=1,
                   psi=None, source=None):
    psi = np.array(sysm.psi if psi is None else psi, dtype=np.float64, copy=True)
    src = np.ascontiguousarray(sysm.source if source is None else source, np.float64)
    lower = sysm.lower_or_upper
    perf = FoamPerf()
    lib().orc_foam_pbicgstab(*_addr(sysm), sysm.diag, sysm.upper, lower, psi, src, tolerance,
                             relTol, maxIter, minIter, nthreads, C.byref(perf))
    return psi, perf


def cg64(sysm, b=None, tol=1e-12, maxIter=200000, transpose=False, nthreads=0, x0=None):
    """FP64 Krylov solve to ||b - A x||_2 <= tol ||b||_2 (accuracy oracle)."""
    if nthreads <= 0:
        nthreads = os.cpu_count() or 1
    b = np.ascontiguousarray(sysm.source if b is None else b, np.float64)
    x = np.zeros(sysm.n) if x0 is None else np.array(x0, np.float64, copy=True)
    it = lib().orc_cg64(*_addr(sysm), sysm.diag, sysm.upper, _ptr_or_none(sysm.lower), x, b,
                        tol, maxIter, int(transpose), nthreads)
    if it < 0:
        raise RuntimeError("cg64 did not reach the requested tolerance")
    return x, it


def face_gradients(sysm, lam, x):
    dU = np.empty(sysm.nf)
    dL = np.empty(sysm.nf)
    dD = np.empty(sysm.n)
    lib().orc_face_gradients(sysm.n, sysm.nf, sysm.addr.lowerAddr, sysm.addr.upperAddr,
                             np.ascontiguousarray(lam, np.float64),
                             np.ascontiguousarray(x, np.float64), dU, dL, dD)
    return dU, dL, dD


def amul_rows(sysm, x, transpose=False, nthreads=1):
    y = np.empty(sysm.n)
    a = sysm.addr
    lib().orc_amul_rows(a.n, a.lowerAddr, a.upperAddr, a.ownerStartAddr, a.losortAddr,
                        a.losortStartAddr, sysm.diag, sysm.upper, _ptr_or_none(sysm.lower),
                        np.ascontiguousarray(x, np.float64), y, int(transpose), nthreads)
    return y


def cheb_constants(order, beta, ratio):
    c = np.zeros(max(2 * order, 2), np.float32)
    lib().orc_cheb_constants(order, beta, ratio, c)
    return c


class Backend:
    """The emulated metalFoamBackend (FP32 inner solves)."""

    def __init__(self, sysm):
        self.sysm = sysm
        self._keep = _addr(sysm)
        self.h = lib().orc_backend_new(*self._keep)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_backend_free(self.h)
            self.h = None

    def set_coeffs(self, diag, upper, lower=None):
        self._c = (np.ascontiguousarray(diag, np.float64), np.ascontiguousarray(upper, np.float64),
                   None if lower is None else np.ascontiguousarray(lower, np.float64))
        lib().orc_backend_set_coeffs(self.h, self._c[0], self._c[1], _ptr_or_none(self._c[2]))

    def pcg(self, r, target, maxIter, iterationsPerSync=1, chebOrder=1, chebBeta=2.0,
            chebRatio=30.0):
        return lib().orc_backend_pcg(self.h, np.ascontiguousarray(r, np.float64), target, maxIter,
                                     iterationsPerSync, chebOrder, chebBeta, chebRatio)

    def bicgstab(self, r, target, maxIter):
        return lib().orc_backend_bicgstab(self.h, np.ascontiguousarray(r, np.float64), target,
                                          maxIter)

    def delta(self):
        p = lib().orc_backend_delta(self.h)
        return np.ctypeslib.as_array(p, shape=(self.sysm.n,)).copy()


# ---------------------------------------------------------------- FP32 kernels

def _f32(a):
    return np.ascontiguousarray(a, np.float32)


class Ldu32View:
    """FP32 copies of a system's coefficients as the reference stages them
    (setCoeffs: float(diag), float(upper), float(lower); rD = float(1/diag))."""

    def __init__(self, sysm, diag=None):
        d = sysm.diag if diag is None else diag
        self.diag = _f32(d)
        self.upper = _f32(sysm.upper)
        self.lower = self.upper if sysm.lower is None else _f32(sysm.lower)
        self.rD = _f32(1.0 / np.asarray(d, np.float64))
        a = sysm.addr
        self.addr = a
        self.s = Ldu32(a.n, a.nf, self.diag.ctypes.data, self.upper.ctypes.data,
                       self.lower.ctypes.data, a.lowerAddr.ctypes.data, a.upperAddr.ctypes.data,
                       a.ownerStartAddr.ctypes.data, a.losortAddr.ctypes.data,
                       a.losortStartAddr.ctypes.data)

    def spmv(self, x, w=None):
        x = _f32(x)
        y = np.empty_like(x)
        if w is None:
            lib().orc_k_ldu_spmv(C.byref(self.s), x, y)
            return y, None
        part = np.zeros((self.addr.n + 255) // 256, np.float32)
        lib().orc_k_ldu_spmv_dotw(C.byref(self.s), x, _f32(w), y, part)
        return y, part

    def cheb_apply(self, r, order, beta, ratio=30.0):
        r = _f32(r)
        n = r.shape[0]
        c = cheb_constants(order, beta, ratio)
        w = np.empty(n, np.float32)
        z = np.empty(n, np.float32)
        v = np.empty(n, np.float32)
        lib().orc_k_cheb_init(n, r, self.rD, w, z, c[0])
        for i in range(1, order):
            lib().orc_k_ldu_spmv(C.byref(self.s), z, v)
            lib().orc_k_cheb_step(n, r, v, self.rD, w, z, c[2 * i - 1], c[2 * i])
        return z


# ------------------------------------------- the reference's kernel sequences
# Slots of the reference's scalar buffer (metalFoamKernels.metal:20-32).
S_ALPHA, S_BETA, S_OMEGA, S_COUNT = 3, 4, 9, 16


def _scalars(alpha=0.0, beta=0.0, omega=0.0):
    s = np.zeros(S_COUNT, np.float32)
    s[S_ALPHA], s[S_BETA], s[S_OMEGA] = alpha, beta, omega
    return s


def _group_count(n):
    return max(1, (n + 255) // 256)


class KernelSequence:
    """One inner iteration's work as the reference dispatches it, kernel by
    kernel (metalFoamBackend.C:608-906), on FP32 copies of a system: each
    method restates what one fused CUDA kernel replaces, with the scalars
    alpha, beta, omega rounded to FP32 as the reference holds them.  Returns
    the vectors the unfused kernels write, plus the FP64 sum of the same FP32
    products that the fused kernel's reduction folds."""

    def __init__(self, sysm):
        self.v = Ldu32View(sysm)
        self.n = sysm.n

    def _spmv(self, x):
        y, _ = self.v.spmv(x)
        return y

    def cheb_step(self, zin, win, rA, order, step, beta, ratio=30.0):
        """ldu_spmv + cheb_step (metalFoamKernels.metal:64-150,174-194)."""
        c = cheb_constants(order, beta, ratio)
        v = self._spmv(zin)
        w, z = _f32(win).copy(), _f32(zin).copy()
        lib().orc_k_cheb_step(self.n, _f32(rA), v, self.v.rD, w, z, c[2 * step - 1], c[2 * step])
        dot = float(np.dot(z.astype(np.float64), _f32(rA).astype(np.float64)))
        return {"wOut": w, "zOut": z}, [dot if step == order - 1 else 0.0, 0.0, 0.0]

    def pcg_p_spmv(self, wA, pOld, beta):
        """pcg_update_p + ldu_spmv_dotw (metalFoamKernels.metal:64-109,237-247)."""
        p = _f32(pOld).copy()
        lib().orc_k_pcg_update_p(self.n, p, _f32(wA), _scalars(beta=beta))
        q = self._spmv(p)
        return {"p": p, "q": q}, [float(np.dot(p.astype(np.float64), q.astype(np.float64))),
                                  0.0, 0.0]

    def pcg_update(self, delta, p, rA, q, alpha, chebOrder=1, chebBeta=2.0, chebRatio=30.0):
        """pcg_update_sol_res, then the next apply: cheb_init (Chebyshev) or
        pcg_precond_dot (Jacobi) (metalFoamKernels.metal:154-171,212-276)."""
        d, r = _f32(delta).copy(), _f32(rA).copy()
        part = np.zeros(_group_count(self.n), np.float32)
        lib().orc_k_pcg_update_sol_res(self.n, d, r, _f32(p), _f32(q), _scalars(alpha=alpha),
                                       part)
        w = np.empty(self.n, np.float32)
        if chebOrder > 1:
            c = cheb_constants(chebOrder, chebBeta, chebRatio)
            z = np.empty(self.n, np.float32)
            lib().orc_k_cheb_init(self.n, r, self.v.rD, w, z, c[0])
            dot = 0.0
        else:
            lib().orc_k_pcg_precond_dot(self.n, r, self.v.rD, w, part)
            dot = float(np.dot(w.astype(np.float64), r.astype(np.float64)))
        l1 = float(np.sum(np.abs(r.astype(np.float64))))
        return {"deltaNext": d, "rAOut": r, "wAOut": w}, [l1, dot, 0.0]

    def bicg_ab(self, rA, pOld, AyAOld, rA0, beta, omega):
        """bicg_update_p, emul, ldu_spmv_dotw (metalFoamKernels.metal:64-109,
        198-208,372-386)."""
        p = _f32(pOld).copy()
        lib().orc_k_bicg_update_p(self.n, p, _f32(rA), _f32(AyAOld),
                                  _scalars(beta=beta, omega=omega))
        y = np.empty(self.n, np.float32)
        lib().orc_k_emul(self.n, self.v.rD, p, y)
        v = self._spmv(y)
        dot = float(np.dot(_f32(rA0).astype(np.float64), v.astype(np.float64)))
        return {"p": p, "yA": y, "AyA": v}, [dot, 0.0, 0.0]

    def bicg_cd(self, rA, AyA, alpha):
        """bicg_s_res, emul, ldu_spmv_dotw, dot_partial (metalFoamKernels.metal:
        64-109,198-208,390-412,280-295)."""
        s = np.empty(self.n, np.float32)
        part = np.zeros(_group_count(self.n), np.float32)
        lib().orc_k_bicg_s_res(self.n, s, _f32(rA), _f32(AyA), _scalars(alpha=alpha), part)
        z = np.empty(self.n, np.float32)
        lib().orc_k_emul(self.n, self.v.rD, s, z)
        t = self._spmv(z)
        s64, t64 = s.astype(np.float64), t.astype(np.float64)
        return {"sA": s, "zA": z, "tA": t}, [float(np.sum(np.abs(s64))), float(np.dot(s64, t64)),
                                             float(np.dot(t64, t64))]

    def bicg_e(self, delta, yA, zA, sA, tA, rA0, alpha, omega):
        """bicg_update_sol_res + dot_partial of rA0.rA (metalFoamKernels.metal:
        280-295,430-458)."""
        d = _f32(delta).copy()
        r = np.empty(self.n, np.float32)
        part = np.zeros(_group_count(self.n), np.float32)
        lib().orc_k_bicg_update_sol_res(self.n, d, _f32(yA), _f32(zA), r, _f32(sA), _f32(tA),
                                        _scalars(alpha=alpha, omega=omega), part)
        r64 = r.astype(np.float64)
        return {"deltaNext": d, "rAOut": r}, [float(np.sum(np.abs(r64))),
                                              float(np.dot(_f32(rA0).astype(np.float64), r64)),
                                              0.0]
