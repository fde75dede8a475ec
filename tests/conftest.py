import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "pyfacc-scf_b200")
for p in (PKG, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

BASIS_DIR = os.path.join(PKG, "data", "basis_set")
MOL_DIR = os.path.join(PKG, "data", "molecules")


def basis_file(name="sto-3g"):
    return os.path.join(BASIS_DIR, f"{name}.txt")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: long-running")


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def engine():
    import pyfacc
    pyfacc.lib()
    return pyfacc
