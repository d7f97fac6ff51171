import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

from ksvd_loader import load, load_oracle  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: long-running case")


@pytest.fixture(scope="session")
def pkg():
    return load()


@pytest.fixture(scope="session")
def oracle():
    o = load_oracle()
    o.lib()
    return o


@pytest.fixture(scope="session")
def ksvd(pkg):
    return pkg.ksvd


@pytest.fixture(scope="session")
def synth(pkg):
    return pkg.synth


@pytest.fixture(scope="session")
def torch_cuda():
    """torch with a CUDA device.  GPU tests fail (not skip) without one."""
    import torch
    assert torch.cuda.is_available(), "GPU test run without a CUDA device"
    return torch


@pytest.fixture(scope="session")
def built_lib(ksvd):
    if not ksvd.LIB_PATH.exists():
        ksvd.build()
    return ksvd.lib()


def rng(seed=0):
    return np.random.default_rng(seed)
