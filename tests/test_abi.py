"""The C-ABI library loads, exports exactly the symbols include/*.h declares, and
its host-side argument and device checks report errors without a GPU."""
import ctypes as C
import glob
import os
import re
import subprocess

import numpy as np

from conftest import ROOT


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        for m in re.finditer(r"MULTIFLOATS_CUDA_API\s+[\w\s\*]+?\b(\w+)\s*\(", src):
            names.add(m.group(1))
    return names


def exported_symbols(path):
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True,
                         check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if re.search(r" [TW] ", line)}


def test_exports_match_header(cuda_lib):
    from multifloats_b200 import _lib

    decl = declared_symbols()
    assert len(decl) >= 30
    exp = exported_symbols(_lib.LIB_PATH)
    assert decl <= exp, f"declared but not exported: {sorted(decl - exp)}"
    extra = {s for s in exp - decl if not s.startswith("_")}
    assert not extra, f"exported but not declared: {sorted(extra)}"


def test_library_loads_and_versions(cuda_lib):
    assert cuda_lib.mfcuda_version().decode().count(".") == 2
    assert cuda_lib.mfcuda_error_string(0) == b"success"


def test_invalid_arguments_rejected_before_device(cuda_lib):
    # negative sizes are rejected by the host-side checks
    rc = cuda_lib.mfcuda_matmuldd_mm(None, None, None, -1, 4, 4, 8, None)
    assert rc == 1
    rc = cuda_lib.mfcuda_unary_dd(0, None, None, -5, None)
    assert rc == 1
    rc = cuda_lib.mfcuda_unary_dd(9, None, None, 0, None)  # unknown op
    assert rc in (1, 4)
    cuda_lib.matmuldd_mm(None, None, None, 3, -2, 3, 8)
    assert cuda_lib.mfcuda_last_error() == 1
    # overflow of m * k is caught
    rc = cuda_lib.mfcuda_matmuldd_mm(None, None, None, 2 ** 40, 2 ** 40, 1, 8, None)
    assert rc == 1


def test_empty_calls_succeed(cuda_lib):
    # m == 0 or n == 0: nothing to do, no device needed
    assert cuda_lib.mfcuda_matmuldd_mm(None, None, None, 0, 5, 7, 8, None) == 0
    assert cuda_lib.mfcuda_unary_dd(0, None, None, 0, None) in (0, 4)


def test_drop_in_without_gpu_latches_error(cuda_lib):
    import torch

    if torch.cuda.is_available():
        return  # covered by the GPU tests
    x = np.zeros(8)
    y = np.zeros(8)
    cuda_lib.expdd_array(x.ctypes.data, y.ctypes.data, 4)
    assert cuda_lib.mfcuda_last_error() == 4  # MFCUDA_ERR_NO_DEVICE
    r = cuda_lib.sumdd_array(x.ctypes.data, 4)
    assert cuda_lib.mfcuda_last_error() == 4
    assert np.isnan(r.hi)


def test_compiled_c_consumer_links_and_reports_no_device():
    """The compiled C caller (tests/consumer/consumer.c, built by
    oracle/Makefile) links against the library alone; without a GPU every
    drop-in latches an error and it exits 2, with one it exits 0."""
    import subprocess

    import torch

    exe = os.path.join(ROOT, "oracle", "_ref", "consumer_c_own")
    if not os.path.exists(exe):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "own-consumer"], check=True)
    proc = subprocess.run([exe, os.devnull], capture_output=True, text=True, timeout=120)
    assert proc.returncode == (0 if torch.cuda.is_available() else 2), (proc.returncode, proc.stderr)
