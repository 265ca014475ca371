"""The OpenFOAM adapter (metal4foam_b200/openfoam/*.C) cannot be built here
(no OpenFOAM); it is compiled with -fsyntax-only against the C ABI header
and a minimal model of the OpenFOAM interfaces it uses
(tests/openfoam_model/), so its calls into include/cudafoam.h are
type-checked and every control key the Python surface accepts is read.
The model includes the processor-interface and Pstream calls the adapter
makes for decomposed cases (cf_subdomain_* with a Pstream cf_comm)."""
import glob
import os
import re
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
ADAPTER = os.path.join(ROOT, "metal4foam_b200", "openfoam")


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
@pytest.mark.parametrize("src", sorted(glob.glob(os.path.join(ADAPTER, "*.C"))),
                         ids=lambda p: os.path.basename(p))
def test_adapter_compiles_against_the_abi(src):
    res = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-Wall", "-Wextra", "-Werror",
                          "-I", os.path.join(HERE, "openfoam_model"),
                          "-I", os.path.join(ROOT, "include"), "-I", ADAPTER, src],
                         capture_output=True, text=True)
    assert res.returncode == 0, res.stderr


def test_adapter_reads_every_control_key():
    from metal4foam_b200.solver import _CONTROL_KEYS
    text = open(os.path.join(ADAPTER, "cudaFoamSolver.C")).read()
    read = set(re.findall(r'getOrDefault<[^>]+>\("([A-Za-z]+)"', text))
    assert set(_CONTROL_KEYS) <= read, sorted(set(_CONTROL_KEYS) - read)


def test_adapter_routes_processor_interfaces_to_subdomains():
    text = open(os.path.join(ADAPTER, "cudaFoamSolver.C")).read()
    for call in ("cf_subdomain_set_topology", "cf_subdomain_set_coeffs", "cf_subdomain_solve",
                 "isA<processorLduInterface>", "interfaceBouCoeffs_[patchi]",
                 "hostBuffers = 1"):
        assert call in text, call
