"""Test configuration: the `gpu` marker and import paths.

`-m "not gpu"` runs on CPU only (oracle checks, host logic, library exports);
`-m gpu` runs the parity tests that call libmoea_b200 on a CUDA device.
"""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / "cuda-moea_b200"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    return O
