import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden", "golden.npz")

# the batch autotuner's cache goes to a per-session temporary file
if "MFCUDA_AUTOTUNE_CACHE" not in os.environ:
    import tempfile

    os.environ["MFCUDA_AUTOTUNE_CACHE"] = os.path.join(tempfile.mkdtemp(prefix="mfcuda_tune_"), "autotune.txt")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (B200)")


@pytest.fixture(scope="session")
def golden():
    return np.load(GOLDEN)


@pytest.fixture(scope="session")
def cuda_lib():
    """The built CUDA library (built in-tree first if it is missing)."""
    from multifloats_b200 import _lib

    if not os.path.exists(_lib.LIB_PATH):
        from multifloats_b200 import build

        build.build()
    return _lib.lib()


@pytest.fixture(scope="session")
def dev():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a visible CUDA device")
    d = torch.device("cuda:0")
    major, _ = torch.cuda.get_device_capability(d)
    if major != 10:
        pytest.fail(f"expected an sm_100 device, got capability {major}.x")
    return d


def to_dev(x, dev):
    import torch

    return torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64)).to(dev)


def to_host(t):
    import torch

    torch.cuda.synchronize()
    return t.cpu().numpy()
