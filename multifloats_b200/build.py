"""Build libmultifloats_cuda.so in-tree with nvcc for sm_100a.

The library is plain CUDA C++ behind a C ABI (include/multifloats_cuda.h); no
PyTorch headers are involved.  Each translation unit is compiled separately
(in parallel), then linked with a static CUDA runtime into
multifloats_b200/libmultifloats_cuda.so.  ptxas resource usage (-Xptxas -v)
is written to multifloats_b200/_build/ptxas.log.

    python -m multifloats_b200.build [--force]
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmultifloats_cuda.so")
PEAKS_LIB = os.path.join(HERE, "libmfcuda_peaks.so")  # bench-only throughput probes

SOURCES = [
    "runtime.cu",
    "elementwise.cu",
    "gemm_dd.cu",
    "reduce_dd.cu",
    "split_gemm.cu",
    "batched.cu",
    "blas_dd.cu",
    "shard.cu",
]
HEADERS = ["common.cuh", "dd_device.cuh", "dd_tables.h", "tcgen05.cuh", "split_device.cuh", "gemm_tile.cuh",
           "crt_device.cuh", "crt_tables.h", "grid_round.cuh"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3",
    "-std=c++17",
    "-lineinfo",
    "--fmad=false",  # no contraction anywhere: the DD algorithms rely on exact roundings
    "-Xptxas", "-v",
    "-Xcompiler", "-fPIC,-fvisibility=hidden,-O2",
    "-I" + os.path.join(ROOT, "include"),
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _deps_mtime(src: str) -> float:
    paths = [os.path.join(CSRC, src)] + [os.path.join(CSRC, h) for h in HEADERS]
    paths.append(os.path.join(ROOT, "include", "multifloats_cuda.h"))
    return max(os.path.getmtime(p) for p in paths if os.path.exists(p))


def _compile(src: str, force: bool) -> tuple[str, str]:
    obj = os.path.join(BUILD, src.replace(".cu", ".o"))
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= _deps_mtime(src):
        log = obj + ".log"
        return obj, open(log).read() if os.path.exists(log) else ""
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-c", os.path.join(CSRC, src), "-o", obj]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{' '.join(cmd)}\n{proc.stdout}\n{proc.stderr}")
    with open(obj + ".log", "w") as f:
        f.write(proc.stderr)
    return obj, proc.stderr


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        results = list(ex.map(lambda s: _compile(s, force), SOURCES))
    objs = [r[0] for r in results]
    with open(os.path.join(BUILD, "ptxas.log"), "w") as f:
        for (obj, log) in results:
            f.write(f"== {os.path.basename(obj)}\n{log}\n")
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        tmp = LIB + ".tmp"
        cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs,
               "-Xcompiler", "-fPIC", "-Xlinker", "--exclude-libs,ALL", "-ldl"]
        proc = subprocess.run(cmd, capture_output=True, text=True)
        if proc.returncode != 0:
            raise RuntimeError(f"link failed:\n{' '.join(cmd)}\n{proc.stdout}\n{proc.stderr}")
        os.replace(tmp, LIB)
    _build_peaks(force)
    if verbose:
        print(open(os.path.join(BUILD, "ptxas.log")).read())
    return LIB


def _build_peaks(force: bool) -> None:
    src = os.path.join(CSRC, "peaks.cu")
    newest = max(os.path.getmtime(src), os.path.getmtime(os.path.join(CSRC, "tcgen05.cuh")))
    if not force and os.path.exists(PEAKS_LIB) and os.path.getmtime(PEAKS_LIB) >= newest:
        return
    cmd = [nvcc(), *ARCH, "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden",
           "-shared", "-cudart", "static", "-o", PEAKS_LIB, src]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"nvcc failed for peaks.cu:\n{proc.stdout}\n{proc.stderr}")


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
