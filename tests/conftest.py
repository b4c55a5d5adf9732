"""Test configuration: import paths and the `gpu` marker.

`-m "not gpu"` runs the oracle pins, host logic and ABI checks on the CPU;
`-m gpu` runs the parity tests through the C ABI on a B200.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for sub in ("oracle", "wqc-core_b200"):
    p = os.path.join(ROOT, sub)
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libwqc_cuda.so")


@pytest.fixture(scope="session")
def cuda_ctx():
    import wqc_cuda

    return wqc_cuda.Context.shared()
