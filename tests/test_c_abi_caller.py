"""The C ABI from a plain C program (tests/c_abi/solve_poisson.c), linked
against libcudafoam.so with gcc: on a machine without an sm_100 device it
must fail cleanly with CF_ERR_NO_DEVICE; on a B200 it must solve to 1e-6 and
its own FP64 residual must match the library's."""
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
PKG = os.path.join(ROOT, "metal4foam_b200")


def build_caller(tmp_path):
    from metal4foam_b200 import _lib
    _lib.load()          # builds libcudafoam.so when absent
    exe = str(tmp_path / "solve_poisson")
    subprocess.run(["gcc", "-O2", "-std=c11", "-I", os.path.join(ROOT, "include"),
                    os.path.join(HERE, "c_abi", "solve_poisson.c"), "-o", exe,
                    "-L", PKG, "-lcudafoam", f"-Wl,-rpath,{PKG}", "-lm"], check=True)
    return exe


def run(exe, *args):
    return subprocess.run([exe, *map(str, args)], capture_output=True, text=True, timeout=300)


def test_c_caller_without_device(tmp_path):
    from conftest import gpu_available
    if gpu_available():
        pytest.skip("a device is present")
    res = run(build_caller(tmp_path), 6, 5, 4)
    assert res.returncode == 3, res.stdout + res.stderr
    assert res.stdout.startswith("status 6")


@pytest.mark.gpu
@pytest.mark.parametrize("precond", ["Chebyshev", "GAMG"])
def test_c_caller_solves(require_gpu, tmp_path, precond):
    res = run(build_caller(tmp_path), 24, 20, 16, precond)
    assert res.returncode == 0, res.stdout + res.stderr
    line = res.stdout.strip().splitlines()[-1].split()
    vals = dict(zip(line[0::2], line[1::2]))
    assert int(vals["converged"]) == 1 and float(vals["final"]) < 1e-6
    assert float(vals["l1"]) / float(vals["normFactor"]) == pytest.approx(float(vals["final"]),
                                                                          rel=1e-6)
