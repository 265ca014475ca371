"""Time the hot kernels of cudaPCG on a synthetic pressure matrix.

    python -m metal4foam_b200.kernel_timing [nx,ny,nz] [reps]
    python -m metal4foam_b200.kernel_timing --batched [count]
    python -m metal4foam_b200.kernel_timing --multi [nx,ny,nz]

Default: builds the seeded variable-coefficient pressure matrix (cells
relabelled by a random permutation), stages it, runs a 2-iteration solve so
every work vector holds finite data, then launches each hot kernel `reps`
times (cf_time_kernel: CUDA events on the context stream) and prints the
average time per launch.  Small enough (<1 GB on the device, ~30 launches
before the timed ones) to run under ncu.

--batched: one batched solve of the first `count` (default 48) systems of
the batched configuration with the host-synchronised loop (graph 0), so a
profiler sees every kernel launch (it cannot see kernel nodes inside graphs
with conditional nodes); prints the solve time and iterations.

--multi: one 3-component cudaPBiCGStab solve of the upwind momentum matrix
(default 64^3) with graph 0, for the same reason.

--gamg: two cudaPCG solves of the pressure matrix (default 128^3) with the
multigrid preconditioner (preconditioner GAMG, defaults), graph 0 -- the
first builds the hierarchy; the second is the one to profile.
"""
from __future__ import annotations

import sys
import time

import numpy as np

from . import _lib, mesh


def single(dims, reps):
    s = mesh.varcoeff3d(dims, seed=1, permute=True)
    ctx = _lib.Context(0)
    a = s.addr
    ctx.set_topology(a.n, a.nf, *a.arrays())
    ctx.set_coeffs(s.diag, s.upper, None)
    psi = np.zeros(s.n)
    ctx.solve(_lib.CF_SOLVER_PCG, psi, s.source, _lib.default_options(maxIter=2))
    for k in ("cheb_step", "spmv32", "pcg_p_spmv", "pcg_update", "amul64"):
        print(f"{k} {ctx.time_kernel(k, reps=reps):.6f} ms/launch", flush=True)
    ctx.close()


def batched(count):
    systems = mesh.batched_systems()[:count]
    bt = _lib.Batch(0)
    for s in systems:
        bt.add_system(s.addr)
    bt.finalize()
    for i, s in enumerate(systems):
        bt.set_coeffs(i, s.diag, s.upper)
    psis = [np.zeros(s.n) for s in systems]
    t0 = time.perf_counter()
    perfs = bt.solve(psis, [s.source for s in systems],
                     _lib.default_options(stagnationLimit=400, maxRestarts=20, maxIter=20000,
                                          graph=0))
    dt = time.perf_counter() - t0
    print(f"batched {len(systems)} systems {sum(s.n for s in systems)} cells: {dt * 1e3:.1f} ms "
          f"(host-synchronised loop), iterations {[p.nIterations for p in perfs]}, "
          f"launches {bt.kernel_launches()}", flush=True)
    bt.close()


def multi(dims):
    s, rhs = mesh.momentum_multi_rhs(dims)
    ctx = _lib.Context(0)
    a = s.addr
    ctx.set_topology(a.n, a.nf, *a.arrays())
    ctx.set_coeffs(s.diag, s.upper, s.lower)
    psi = np.zeros_like(rhs)
    t0 = time.perf_counter()
    perfs = ctx.solve_multi(_lib.CF_SOLVER_PBICGSTAB, psi, np.ascontiguousarray(rhs),
                            _lib.default_options(graph=0))
    dt = time.perf_counter() - t0
    print(f"multi-RHS {dims} x {rhs.shape[0]}: {dt * 1e3:.1f} ms (host-synchronised loop), "
          f"iterations {[p.nIterations for p in perfs]}", flush=True)
    ctx.close()


def gamg(dims):
    s = mesh.varcoeff3d(dims, seed=1, permute=True)
    ctx = _lib.Context(0)
    a = s.addr
    ctx.set_topology(a.n, a.nf, *a.arrays())
    ctx.set_coeffs(s.diag, s.upper, None)
    opts = _lib.default_options(preconditioner="GAMG", graph=0, profile=True)
    for k in range(2):
        psi = np.zeros(s.n)
        t0 = time.perf_counter()
        p = ctx.solve(_lib.CF_SOLVER_PCG, psi, s.source, opts)
        dt = time.perf_counter() - t0
        print(f"GAMG solve {k} {dims}: {dt * 1e3:.1f} ms (host-synchronised loop), iterations "
              f"{p.nIterations}, final residual {p.finalResidual:.3e}, levels "
              f"{ctx.gamg_levels()}", flush=True)
    ctx.close()


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    if argv and argv[0] == "--batched":
        batched(int(argv[1]) if len(argv) > 1 else 48)
        return
    if argv and argv[0] == "--gamg":
        gamg(tuple(int(x) for x in (argv[1] if len(argv) > 1 else "128,128,128").split(",")))
        return
    if argv and argv[0] == "--multi":
        multi(tuple(int(x) for x in (argv[1] if len(argv) > 1 else "64,64,64").split(",")))
        return
    dims = tuple(int(x) for x in (argv[0] if argv else "128,128,128").split(","))
    reps = int(argv[1]) if len(argv) > 1 else 3
    single(dims, reps)


if __name__ == "__main__":
    main()
