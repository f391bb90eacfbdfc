"""pytest configuration: marker registration and import paths.

``-m "not gpu"`` runs everywhere (oracle pins, golden vectors, host logic, ABI surface);
``-m gpu`` needs a CUDA device and calls the library through its C ABI.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "sma-dft_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device; calls libsmadft.so through the C ABI")


@pytest.fixture(scope="session")
def smadft_lib():
    """The product library (built in place if missing: there is no CPU fallback)."""
    import smadft
    if not os.path.exists(smadft.LIB_PATH):
        smadft.build()
    return smadft.lib()
