"""Iterations the reference's CPU path needs on the bench workload.

The CPU path the plugin mirrors is OpenFOAM's FP64 PCG (oracle/foam_cpu.c
restates it).  A full solve of the 128^3 permuted pressure matrix to FP64
normalised residual 1e-6 takes minutes, so bench.py times bounded samples
(seconds per iteration on the host it runs on) and multiplies by the
iteration counts this script measures (they depend only on the matrix and
the arithmetic, not on the host):

    python oracle/cpu_baseline_iterations.py
    -> DIC (serial): 769 iterations; diagonal: 1717 iterations

(measured with this script; the values are recorded in bench.py).
"""
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def main():
    from metal4foam_b200 import mesh
    from oracle import oracle as O
    s = mesh.varcoeff3d((128, 128, 128), seed=1, permute=True)
    for pre, nt in (("DIC", 1), ("diagonal", os.cpu_count() or 1)):
        t0 = time.time()
        _, p = O.foam_pcg(s, pre, tolerance=1e-6, maxIter=20000, nthreads=nt)
        print(f"{pre}: {p.nIterations} iterations, final residual {p.finalResidual:.3e}, "
              f"converged {bool(p.converged)}, {time.time() - t0:.1f} s with {nt} threads",
              flush=True)


if __name__ == "__main__":
    main()
