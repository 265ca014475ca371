"""Generate tests/golden/headline_reference.json: what the reference
algorithm does on the two full-size single-system configurations.

The oracle's metal_solve restates the reference's FP64 driver
(metalFoamSolver.C:77-437) around its FP32 inner solves
(metalFoamBackend.C:568-959, kernels metalFoamKernels.metal emulated op by
op in IEEE FP32).  At full size it runs single-threaded for minutes, longer
than a GPU test may take, so its outcome is recorded here once:

  * the 128^3 variable-coefficient pressure system (seed 1, cells permuted),
    cudaPCG defaults (Chebyshev order 8, deflate auto, maxRestarts 8,
    tolerance 1e-6);
  * the 96^3 upwind convection-diffusion system (seed 2), PBiCGStab,
    tolerance 1e-8, maxIter 5000.

tests/test_gpu_headline.py compares the CUDA solves with these outcomes and
with an FP64 solve computed in the test itself.

  python tests/golden/make_headline_golden.py
"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from metal4foam_b200 import mesh  # noqa: E402
from oracle import oracle as O  # noqa: E402

OUT = os.path.join(HERE, "headline_reference.json")


def record(r, seconds):
    return {"nIterations": r.nIterations, "nRestarts": r.nRestarts,
            "initialResidual": r.initialResidual, "finalResidual": r.finalResidual,
            "converged": r.converged, "singular": r.singular, "deflated": r.deflated,
            "polished": r.polished, "chebBeta": r.chebBeta, "normFactor": r.normFactor,
            "seconds_single_thread": round(seconds, 1)}


def main():
    out = {}
    s = mesh.varcoeff3d((128, 128, 128), seed=1, permute=True)
    t0 = time.perf_counter()
    r = O.metal_solve(s)
    out["varcoeff128_pcg"] = dict(record(r, time.perf_counter() - t0),
                                  controls={"chebyshevOrder": 8, "deflate": "auto",
                                            "maxRestarts": 8, "tolerance": 1e-6})
    s = mesh.upwind3d((96, 96, 96), seed=2)
    t0 = time.perf_counter()
    r = O.metal_solve(s, bicgstab=True, tolerance=1e-8, maxIter=5000)
    out["upwind96_pbicgstab"] = dict(record(r, time.perf_counter() - t0),
                                     controls={"tolerance": 1e-8, "maxIter": 5000})
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
        f.write("\n")
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
