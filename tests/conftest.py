"""Shared test set-up. Tests marked `gpu` need a CUDA device and the built libcspb.so; every other test runs on the
CPU (the oracle, the host logic, the C ABI's exports and argument checks)."""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libcspb.so")


@pytest.fixture(scope="session")
def cuda():
    """The CUDA device. On a machine with a GPU the library MUST load (no silent fallback)."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import cospanmdao_b200 as cb
    cb.lib()  # raises LibraryMissing when the CUDA library is not built
    return torch.device("cuda", 0)


@pytest.fixture(scope="session")
def golden():
    import numpy as np
    d = ROOT / "tests" / "golden"

    def load(name):
        return dict(np.load(d / name))
    return load
