"""Compiled C and C++ callers of the drop-in boundary (tests/consumer/consumer.c,
built by oracle/Makefile): the library header alone, and the reference's own
header included first (its MULTIFLOATS_ABI_VERSION makes the library header
reuse the reference's structs; in C++ they live in namespace multifloats)
with -lmultifloats_cuda linked ahead of the reference library.  The programs
call matmuldd_mm, expdd_array and dotdd_array with host pointers; their
outputs must equal the oracle bit for bit, matmuldd_mm must be bound to this
library and the scalar expdd to the reference's, and expdd_array must equal
the reference's scalar expdd element by element in the same process."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from oracle import oracle as O

pytestmark = pytest.mark.gpu

BIN = os.path.join(ROOT, "oracle", "_ref")


def _run(name, tmp_path):
    exe = os.path.join(BIN, name)
    if name != "consumer_c_own" and not O.ref_available():
        pytest.skip("reference library not built here")
    assert os.path.exists(exe), f"{exe} missing: run `make -C oracle consumers`"
    out = tmp_path / f"{name}.bin"
    proc = subprocess.run([exe, str(out)], capture_output=True, text=True, timeout=300)
    assert proc.returncode == 0, (proc.returncode, proc.stdout, proc.stderr)
    return proc.stdout, np.fromfile(str(out), dtype=np.float64)


@pytest.mark.parametrize("name", ["consumer_c_own", "consumer_c_ref", "consumer_cxx_ref"])
def test_compiled_consumer(name, tmp_path):
    text, raw = _run(name, tmp_path)
    assert "matmuldd_mm from libmultifloats_cuda.so" in text, text
    assert "expdd_array from libmultifloats_cuda.so" in text, text
    if name != "consumer_c_own":
        assert "expdd from libmfref.so" in text, text
        assert "scalar expdd matches expdd_array: 4096 / 4096" in text, text
    m, k, n, nx = (int(v) for v in raw[:4].view(np.int64))
    off = 4
    parts = {}
    for key, cnt in (("a", m * k), ("b", k * n), ("c", m * n), ("x", nx), ("y", nx), ("w", nx), ("d", 1)):
        parts[key] = raw[off: off + 2 * cnt]
        off += 2 * cnt
    assert off == raw.size
    assert O.same_bits(parts["c"], O.matmul_mm(parts["a"], parts["b"], m, k, n, 8)).all()
    assert O.same_bits(parts["y"], O.unary("exp", parts["x"])).all()
    assert O.same_bits(parts["d"], O.reduce_blocked("dot", parts["x"], parts["w"], 8)).all()
