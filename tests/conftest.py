"""Test configuration: the `gpu` marker and shared fixtures.

`pytest -m "not gpu"` runs here without a GPU (oracle vs LAPACK / golden
fixtures, host logic, C-ABI exports).  `pytest -m gpu` runs on a B200 and
checks the CUDA path, called through the C ABI, against the oracle.
"""
import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def evdlib():
    """The built C-ABI library (built on first use if absent)."""
    from evd4sc2025_b200 import build as _build
    if not _build.LIB.exists():
        _build.build()
    import evd4sc2025_b200 as evd
    evd.lib()
    return evd


@pytest.fixture(scope="session")
def cuda(evdlib):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a CUDA device")
    return torch.device("cuda:0")
