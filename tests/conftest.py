import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (B200)")


_GPU = None


def gpu_available():
    global _GPU
    if _GPU is None:
        try:
            from metal4foam_b200 import _lib
            ctx = _lib.Context(0)
            ctx.close()
            _GPU = True
        except Exception as e:  # no device here: CPU container
            _GPU = str(e)
    return _GPU is True


@pytest.fixture(scope="session")
def require_gpu():
    if not gpu_available():
        pytest.skip(f"no sm_100 device: {_GPU}")
    return True


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.lib()
    return O
