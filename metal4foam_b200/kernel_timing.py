"""Time the hot kernels of cudaPCG on a synthetic pressure matrix.

    python -m metal4foam_b200.kernel_timing [nx,ny,nz] [reps]

Builds the seeded variable-coefficient pressure matrix (cells relabelled by
a random permutation), stages it, runs a 2-iteration solve so every work
vector holds finite data, then launches each hot kernel `reps` times
(cf_time_kernel: CUDA events on the context stream) and prints the average
time per launch.  Small enough (<1 GB on the device, ~30 launches before the
timed ones) to run under ncu.
"""
from __future__ import annotations

import sys

import numpy as np

from . import _lib, mesh


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    dims = tuple(int(x) for x in (argv[0] if argv else "128,128,128").split(","))
    reps = int(argv[1]) if len(argv) > 1 else 3
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


if __name__ == "__main__":
    main()
