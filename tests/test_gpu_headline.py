"""Parity at the full-size single-system configurations.

* 128^3 variable-coefficient pressure system, cells permuted (2,097,152
  cells, 6,242,304 faces), solved through the cudaPCG plugin surface with
  its defaults to tolerance 1e-6 -- the benchmark's headline system;
* 96^3 first-order upwind convection-diffusion system (884,736 cells),
  cudaPBiCGStab to tolerance 1e-8.

For each: the FP64 normalised residual of the returned psi is recomputed on
the CPU (the oracle's OpenFOAM Amul and normFactor, metalFoamSolver.C:
109-128); the solution is compared with an FP64 solve of the same system
converged to 1e-12; the driver's decisions and iteration counts are compared
with what the reference algorithm does on the same system
(tests/golden/headline_reference.json, recorded by
tests/golden/make_headline_golden.py from the oracle's restatement of
metalFoamSolver.C:77-437 around the emulated FP32 kernels).
"""
import json
import os

import numpy as np
import pytest

from metal4foam_b200 import mesh
from metal4foam_b200.solver import backend_cache_clear, lduMatrix

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                      "headline_reference.json")


def golden(key):
    with open(GOLDEN) as f:
        return json.load(f)[key]


def fp64_residual(oracle, s, psi):
    """sum|b - A psi| / normFactor with the factor of psi0 = 0."""
    z = np.zeros(s.n)
    nf = oracle.normfactor(z, s.source, oracle.amul(s, z), oracle.sumA(s))
    return float(np.sum(np.abs(s.source - oracle.amul(s, psi))) / nf)


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def test_headline_128_cubed_pcg(require_gpu, oracle):
    s = mesh.varcoeff3d((128, 128, 128), seed=1, permute=True)
    m = lduMatrix(s.addr, s.diag, s.upper)
    solver = lduMatrix.solver.New("p", m, {"solver": "cudaPCG", "tolerance": 1e-6,
                                           "relTol": 0.0})
    psi = np.zeros(s.n)
    perf = solver.solve(psi, s.source)
    backend_cache_clear()
    assert perf.converged and perf.finalResidual < 1e-6
    # the residual the driver reports is the FP64 residual of psi
    res = fp64_residual(oracle, s, psi)
    assert res < 1e-6
    assert res == pytest.approx(perf.finalResidual, rel=1e-9)
    # the reference algorithm on the same system: same deflation decision,
    # converged too, iterations within 10%
    ref = golden("varcoeff128_pcg")
    assert ref["converged"] and perf.deflated == ref["deflated"]
    assert abs(perf.nIterations - ref["nIterations"]) <= max(2, 0.10 * ref["nIterations"]), (
        perf.nIterations, ref["nIterations"])
    assert perf.initialResidual == pytest.approx(ref["initialResidual"], rel=1e-12)
    # error against an FP64 PCG solve converged to normalised residual 1e-12
    x64, p64 = oracle.foam_pcg(s, "diagonal", tolerance=1e-12, maxIter=10000,
                               nthreads=host_threads())
    assert p64.finalResidual < 1e-12
    err = float(np.max(np.abs(psi - x64)) / np.max(np.abs(x64)))
    assert err <= 1e-5, err


def test_upwind_96_cubed_pbicgstab(require_gpu, oracle):
    s = mesh.upwind3d((96, 96, 96), seed=2)
    m = lduMatrix(s.addr, s.diag, s.upper, s.lower)
    solver = lduMatrix.solver.New("U", m, {"solver": "cudaPBiCGStab", "tolerance": 1e-8,
                                           "relTol": 0.0, "maxIter": 5000})
    psi = np.zeros(s.n)
    perf = solver.solve(psi, s.source)
    backend_cache_clear()
    assert perf.converged and perf.finalResidual < 1e-8
    res = fp64_residual(oracle, s, psi)
    assert res < 1e-8
    assert res == pytest.approx(perf.finalResidual, rel=1e-9)
    x64, it = oracle.cg64(s, tol=1e-12, nthreads=host_threads())
    err = float(np.max(np.abs(psi - x64)) / np.max(np.abs(x64)))
    assert err <= 1e-7, err
    # the reference algorithm breaks down here: its FP32 fold of rA0.rA
    # reaches exactly 0 and the next scalars are not finite (the documented
    # deviation: FP64-accumulated reductions)
    ref = golden("upwind96_pbicgstab")
    assert ref["singular"] and not ref["converged"] and ref["finalResidual"] > 1e-2
