"""Decomposed solves on the GPU: subdomains with processor interfaces
(cf_subdomain_*), the subdomains of one case solved by threads of one
process on one GPU through the in-process communicator
(cf_comm_local_create; the kernels never wait on one another, the host
threads meet at barriers).

* One subdomain without interfaces returns bit for bit what cf_solve
  returns (same kernels' arithmetic, same grids, identity communication).
* Two to four subdomains (slabs, and a random split that puts most faces on
  interfaces): the assembled psi reaches the tolerance by the FP64 residual
  of the UNSPLIT system recomputed on the CPU (the oracle's Amul and
  normFactor), agrees with an FP64 solve of the unsplit system, and takes
  within 10% (+2) of the iterations of the unsplit cudaPCG/cudaPBiCGStab
  solve (only the order of the global sums differs).
* A subdomain whose interface does not match its neighbour's fails, and so
  does every other subdomain -- none waits for ever.
"""
import threading

import numpy as np
import pytest

from metal4foam_b200 import _lib, decompose, mesh

pytestmark = pytest.mark.gpu


def solve_decomposed(s, part, k, solver, timeout=120.0, **kw):
    subs = decompose.decompose(s, part, k)
    solvers = [_lib.SubdomainSolver(sd) for sd in subs]
    comm = _lib.LocalComm(k, timeout)
    opts = _lib.default_options(**kw)
    psis = [np.zeros(sd.n) for sd in subs]
    perfs, errs = [None] * k, [None] * k

    def run(r):
        try:
            perfs[r] = solvers[r].solve(solver, psis[r], subs[r].system.source, opts, comm[r])
        except Exception as e:  # noqa: BLE001
            errs[r] = e

    th = [threading.Thread(target=run, args=(r,)) for r in range(k)]
    for t in th:
        t.start()
    for t in th:
        t.join(600)
    assert not any(t.is_alive() for t in th)
    for sv in solvers:
        sv.close()
    comm.close()
    return subs, psis, perfs, errs


def fp64_residual(oracle, s, psi):
    z = np.zeros(s.n)
    nf = oracle.normfactor(z, s.source, oracle.amul(s, z), oracle.sumA(s))
    return float(np.sum(np.abs(s.source - oracle.amul(s, psi))) / nf)


def unsplit_solve(s, solver, **kw):
    ctx = _lib.Context(0)
    a = s.addr
    ctx.set_topology(a.n, a.nf, *a.arrays())
    ctx.set_coeffs(s.diag, s.upper, s.lower)
    x = np.zeros(s.n)
    p = ctx.solve(solver, x, s.source, _lib.default_options(**kw))
    ctx.close()
    return x, p


FIELDS = ("initialResidual", "finalResidual", "nIterations", "nRestarts", "converged",
          "singular", "stagnated", "deflated", "polished", "normFactor", "finalResSum32",
          "residualL2", "chebBeta")

ONE = [
    ("varcoeff_cheb8", lambda: mesh.varcoeff3d((40, 40, 40), seed=4, permute=True),
     _lib.CF_SOLVER_PCG, dict()),
    ("varcoeff_jacobi", lambda: mesh.varcoeff3d((30, 28, 25), seed=5),
     _lib.CF_SOLVER_PCG, dict(chebyshevOrder=1, maxIter=3000)),
    ("upwind_bicgstab", lambda: mesh.upwind3d((30, 28, 26), seed=6),
     _lib.CF_SOLVER_PBICGSTAB, dict(tolerance=1e-8, maxIter=3000)),
]


@pytest.mark.parametrize("name,make,solver,kw", ONE, ids=[c[0] for c in ONE])
def test_one_subdomain_equals_single_solve(require_gpu, name, make, solver, kw):
    s = make()
    # cf_solve would take meshes of <= 16384 cells into the cluster path
    kw = dict(kw, clusterMaxCells=-1)
    x_ref, p_ref = unsplit_solve(s, solver, **kw)
    subs, psis, perfs, errs = solve_decomposed(s, np.zeros(s.n, np.int32), 1, solver, **kw)
    assert errs == [None], errs
    for f in FIELDS:
        assert getattr(perfs[0], f) == getattr(p_ref, f), (f, getattr(perfs[0], f),
                                                           getattr(p_ref, f))
    assert np.array_equal(psis[0], x_ref)


SPLITS = [
    ("pcg_slabs2", lambda: mesh.varcoeff3d((36, 34, 32), seed=7), "slab", 2,
     _lib.CF_SOLVER_PCG, dict(), 1e-6),
    ("pcg_slabs4", lambda: mesh.varcoeff3d((36, 34, 32), seed=7), "slab", 4,
     _lib.CF_SOLVER_PCG, dict(), 1e-6),
    ("pcg_random3_permuted", lambda: mesh.varcoeff3d((30, 30, 30), seed=8, permute=True),
     "random", 3, _lib.CF_SOLVER_PCG, dict(), 1e-6),
    ("pcg_jacobi_slabs2", lambda: mesh.poisson2d(120, 110, seed=9), "slab", 2,
     _lib.CF_SOLVER_PCG, dict(chebyshevOrder=1, maxIter=5000), 1e-6),
    ("bicgstab_slabs2", lambda: mesh.upwind3d((32, 30, 28), seed=10), "slab", 2,
     _lib.CF_SOLVER_PBICGSTAB, dict(tolerance=1e-8, maxIter=3000), 1e-8),
    ("bicgstab_random2", lambda: mesh.upwind3d((24, 22, 20), seed=11), "random", 2,
     _lib.CF_SOLVER_PBICGSTAB, dict(tolerance=1e-8, maxIter=3000), 1e-8),
]


@pytest.mark.parametrize("name,make,kind,k,solver,kw,tol", SPLITS, ids=[c[0] for c in SPLITS])
def test_decomposed_matches_unsplit(require_gpu, oracle, name, make, kind, k, solver, kw, tol):
    s = make()
    part = (decompose.slab_partition(s.n, k) if kind == "slab"
            else np.random.default_rng(3).integers(0, k, s.n).astype(np.int32))
    subs, psis, perfs, errs = solve_decomposed(s, part, k, solver, **kw)
    assert errs == [None] * k, errs
    x = decompose.assemble(subs, s.n, psis)
    # every subdomain saw the same global quantities and decisions
    for f in ("initialResidual", "finalResidual", "nIterations", "nRestarts", "deflated",
              "normFactor", "chebBeta", "converged"):
        assert len({getattr(p, f) for p in perfs}) == 1, f
    p = perfs[0]
    assert p.converged and p.finalResidual < tol
    res = fp64_residual(oracle, s, x)
    assert res < tol
    assert res == pytest.approx(p.finalResidual, rel=1e-6)
    x_ref, p_ref = unsplit_solve(s, solver, **kw)
    assert p.deflated == p_ref.deflated
    assert abs(p.nIterations - p_ref.nIterations) <= max(2, 0.10 * p_ref.nIterations), (
        p.nIterations, p_ref.nIterations)
    x64, _ = oracle.cg64(s, tol=1e-12)
    err = float(np.max(np.abs(x - x64)) / np.max(np.abs(x64)))
    assert err < (1e-5 if tol >= 1e-6 else 1e-7), err


def test_mismatched_interface_fails_every_subdomain(require_gpu):
    """Subdomain 1 is told its interface has one face fewer than subdomain
    0's: the exchange finds no matching interface, the failing subdomain
    aborts the in-process hub, and both solves return an error within the
    hub's time limit instead of waiting."""
    s = mesh.varcoeff3d((20, 18, 16), seed=12)
    subs = decompose.decompose(s, decompose.slab_partition(s.n, 2), 2)
    itf = subs[1].interfaces[0]
    itf.faceCells = itf.faceCells[:-1]
    itf.coeffs = itf.coeffs[:-1]
    solvers = [_lib.SubdomainSolver(sd) for sd in subs]
    comm = _lib.LocalComm(2, 20.0)
    opts = _lib.default_options()
    errs = [None, None]

    def run(r):
        try:
            solvers[r].solve(_lib.CF_SOLVER_PCG, np.zeros(subs[r].n), subs[r].system.source,
                             opts, comm[r])
        except Exception as e:  # noqa: BLE001
            errs[r] = e

    th = [threading.Thread(target=run, args=(r,)) for r in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join(120)
    assert not any(t.is_alive() for t in th)
    assert all(isinstance(e, _lib.CudaFoamError) for e in errs), errs
    # the subdomain objects stay usable: a consistent pair solves afterwards
    subs2, psis, perfs, errs2 = solve_decomposed(s, decompose.slab_partition(s.n, 2), 2,
                                                 _lib.CF_SOLVER_PCG)
    assert errs2 == [None, None] and perfs[0].converged
    for sv in solvers:
        sv.close()
    comm.close()


class _HostThreadsComm:
    """cf_comm with host buffers (hostBuffers = 1), written in Python for
    the subdomains of one process: the form an MPI (Pstream) caller
    without CUDA awareness uses.  Sums fold in rank order, as the
    in-process hub's do."""

    def __init__(self, k, subs):
        import ctypes as C
        self.k = k
        self.bar = threading.Barrier(k, timeout=60)
        self.vals = [None] * k
        self.sends = [None] * k
        self.comms = []
        for r in range(k):
            def allreduce(user, values, count, op, stream, r=r):
                try:
                    v = np.ctypeslib.as_array((C.c_double * count).from_address(values))
                    self.vals[r] = v.copy()
                    self.bar.wait()
                    out = self.vals[0].copy()
                    for q in range(1, k):
                        out = np.maximum(out, self.vals[q]) if op == 1 else out + self.vals[q]
                    self.bar.wait()
                    v[:] = out
                    return 0
                except Exception:  # noqa: BLE001
                    return 1

            def exchange(user, nif, nb, nfc, eb, send, recv, stream, r=r):
                try:
                    ct = C.c_double if eb == 8 else C.c_float
                    nbs = np.ctypeslib.as_array((C.c_int32 * nif).from_address(nb))
                    nfs = np.ctypeslib.as_array((C.c_int32 * nif).from_address(nfc))
                    sp = (C.c_void_p * nif).from_address(send)
                    rp = (C.c_void_p * nif).from_address(recv)
                    self.sends[r] = {int(nbs[p]): np.ctypeslib.as_array(
                        (ct * int(nfs[p])).from_address(sp[p])).copy() for p in range(nif)}
                    self.bar.wait()
                    for p in range(nif):
                        got = self.sends[int(nbs[p])][r]
                        np.ctypeslib.as_array((ct * int(nfs[p])).from_address(rp[p]))[:] = got
                    self.bar.wait()
                    return 0
                except Exception:  # noqa: BLE001
                    return 1

            cbs = (_lib.ALLREDUCE_FN(allreduce), _lib.EXCHANGE_FN(exchange),
                   _lib.ABORT_FN(lambda user: self.bar.abort()))
            self.comms.append((_lib.Comm(None, cbs[0], cbs[1], cbs[2], 1), cbs))

    def __getitem__(self, r):
        return self.comms[r][0]


def test_host_buffer_communication_equals_device(require_gpu):
    """The same decomposed solve with the in-process hub (device buffers)
    and with a host-buffer communicator: bit-identical results."""
    s = mesh.varcoeff3d((28, 26, 24), seed=13)
    part = decompose.slab_partition(s.n, 2)
    subs, psis_dev, perfs_dev, errs = solve_decomposed(s, part, 2, _lib.CF_SOLVER_PCG)
    assert errs == [None, None]
    solvers = [_lib.SubdomainSolver(sd) for sd in subs]
    comm = _HostThreadsComm(2, subs)
    opts = _lib.default_options()
    psis = [np.zeros(sd.n) for sd in subs]
    perfs, errs = [None, None], [None, None]

    def run(r):
        try:
            perfs[r] = solvers[r].solve(_lib.CF_SOLVER_PCG, psis[r], subs[r].system.source, opts,
                                        comm[r])
        except Exception as e:  # noqa: BLE001
            errs[r] = e

    th = [threading.Thread(target=run, args=(r,)) for r in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join(600)
    assert errs == [None, None], errs
    for r in range(2):
        assert np.array_equal(psis[r], psis_dev[r])
        assert perfs[r].nIterations == perfs_dev[r].nIterations
        assert perfs[r].finalResidual == perfs_dev[r].finalResidual
    for sv in solvers:
        sv.close()
