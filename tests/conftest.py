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


def wgemm_golden(golden):
    """(case index, args for wgemm(...), expected C) for every stored wgemm case;
    args = (transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)."""
    i = 0
    while f"wgemm{i}_p" in golden.files:
        p = golden[f"wgemm{i}_p"]
        m, n, k, lda, ldb, ldc = (int(v) for v in p[2:])
        s = golden[f"wgemm{i}_s"]
        yield i, (chr(p[0]), chr(p[1]), m, n, k, s[:2], golden[f"wgemm{i}_a"], lda,
                  golden[f"wgemm{i}_b"], ldb, s[2:], golden[f"wgemm{i}_c"], ldc), golden[f"wgemm{i}_out"]
        i += 1


def wtrsm_golden(golden):
    """(case index, args for wtrsm(...), expected B) for every stored wtrsm case;
    args = (side, uplo, transa, diag, m, n, alpha, a, lda, b, ldb)."""
    i = 0
    while f"wtrsm{i}_p" in golden.files:
        p = golden[f"wtrsm{i}_p"]
        m, n, lda, ldb = (int(v) for v in p[4:])
        yield i, (chr(p[0]), chr(p[1]), chr(p[2]), chr(p[3]), m, n, golden[f"wtrsm{i}_s"],
                  golden[f"wtrsm{i}_a"], lda, golden[f"wtrsm{i}_b"], ldb), golden[f"wtrsm{i}_out"]
        i += 1
