#!/usr/bin/env python3
"""Benchmark of the DD GEMM hot path on B200: DD-GFLOP/s at M=N=K=4096.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload gemm4096|gemm256|elementwise|reduce]

One step = one C = A*B of 4096^3 real64x2 operands resident in HBM (each
operand is 256 MiB, larger than the 126 MB L2, so no flush is needed between
steps).  DD-GFLOP/s = 2*M*N*K / seconds / 1e9.  With N GPUs (one process per
GPU under torchrun) every rank multiplies its own independent pair of
matrices (weak scaling, no collective on the data path); the timed region is
bracketed by a barrier and a device synchronise, and the time is the max over
ranks.  Rank 0 prints one JSON line.

--impl reference times the reference library's own CPU matmuldd_mm (built from
the reference sources into oracle/_ref/, else the C restatement in oracle/)
on all host cores, each step a bounded sample of the same workload (a block of
columns of B and C), and prints the same metric.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

M = N = K = 4096
RI = 8
FP64_INSTR_PER_MAC = 13 + 6 / RI  # mac_inl (matmul.inc:6-19) + renorm_inl every RI steps
METRIC = "DD-GEMM DD-GFLOP/s 4096^3: split-INT8 vs plain FP64-DD, 1 B200, err<=8 DD ulp"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# --------------------------------------------------------------------------- env
def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch.distributed as dist

        backend = "nccl"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(ws, value: float) -> float:
    if ws == 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ------------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str | None):
        self.gpu_id = gpu_id
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"]
        if self.gpu_id:
            cmd += ["-i", self.gpu_id]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.reader = threading.Thread(target=self._read, daemon=True)
            self.reader.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.reader.join(timeout=2)

    def summary(self) -> dict:
        sm, mx, reasons, power = [], 0.0, set(), []
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
                power.append(float(parts[3]))
            except ValueError:
                continue
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "power_w_max": max(power) if power else None}


def gpu_uuid() -> str | None:
    try:
        import torch

        u = torch.cuda.get_device_properties(torch.cuda.current_device()).uuid
        return "GPU-" + str(u)
    except Exception:
        return None


def measured_peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return json.load(open(p))
    return {}


# ------------------------------------------------------------------ CPU baseline
def cpu_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_gemm_sample(target_s: float, threads: int):
    """Time the reference CPU matmuldd_mm (or the oracle port) on a block of
    columns of the 4096^3 workload sized to take about target_s seconds."""
    from multifloats_b200 import workloads as W
    from oracle import oracle as O

    kind = "reference" if O.ref_available() else "port"
    A = W.dd_rowcol_scaled(M, K, 16, "row", seed=1)
    Bfull = W.dd_rowcol_scaled(K, 64, 16, "col", seed=2)

    def run(nb):
        Bs = Bfull[: 2 * K * nb]
        t0 = time.perf_counter()
        if kind == "reference":
            O.ref_matmul_mm(A, Bs, M, K, nb, RI, threads=threads)
        else:
            O.matmul_mm(A, Bs, M, K, nb, RI)
        return time.perf_counter() - t0

    nb = max(2, 2 * threads) if kind == "reference" else 2
    nb = min(nb, 64)
    dt = run(nb)
    rate = 2.0 * M * K * nb / dt
    want_nb = int(rate * target_s / (2.0 * M * K))
    want_nb = max(2, min(want_nb - want_nb % 2, 4096))
    Bfull = W.dd_rowcol_scaled(K, want_nb, 16, "col", seed=2) if want_nb > 64 else Bfull
    return kind, want_nb, lambda: run(want_nb)


# --------------------------------------------------------------------- GPU arm
def run_ours(args, ws, rank, local):
    import torch

    from multifloats_b200 import _lib, api
    from multifloats_b200 import workloads as W

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    L = _lib.lib()
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)

    # cpu baseline first (rank 0, N = 1 only) so it never overlaps GPU timing
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        threads = cpu_threads()
        kind, nb, fn = cpu_gemm_sample(args.cpu_seconds, threads)
        dt = fn()
        cpu = {"value": 2.0 * M * K * nb / dt / 1e9, "unit": "DD-GFLOP/s", "cores": threads,
               "kind": kind,
               "sample": f"matmuldd_mm on A 4096x4096 times B 4096x{nb} (columns of the 4096^3 "
                         f"workload), ri={RI}, {threads} threads, {dt:.1f} s"}
        log("cpu baseline:", cpu)

    # operands: per-row / per-column exponent ranges R=16 (split config) -- both forms see the same data
    A = W.dd_rowcol_scaled(M, K, 16, "row", seed=10 + rank)
    B = W.dd_rowcol_scaled(K, N, 16, "col", seed=20 + rank)
    dA = torch.from_numpy(A).to(dev)
    dB = torch.from_numpy(B).to(dev)
    dC = torch.empty(2 * M * N, dtype=torch.float64, device=dev)

    def plain_step():
        _lib.check(L.mfcuda_matmuldd_mm(dA.data_ptr(), dB.data_ptr(), dC.data_ptr(), M, K, N, RI, sp),
                   "mfcuda_matmuldd_mm")

    # FP64 pipe peak (own probe, same process, just before timing)
    peak_lib = C.CDLL(os.path.join(ROOT, "multifloats_b200", "libmfcuda_peaks.so"))
    peak_lib.mfpeak_fp64.argtypes = [C.c_int64, C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    ms_p, ins_p = C.c_double(), C.c_double()
    peak_lib.mfpeak_fp64(200000, sp, C.byref(ms_p), C.byref(ins_p))
    fp64_peak_instr = ins_p.value / (ms_p.value * 1e-3)

    for _ in range(args.warmup):
        plain_step()
    torch.cuda.synchronize()
    barrier(ws)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(gpu_uuid()) as clk:
        torch.cuda.synchronize()
        barrier(ws)
        e0.record(stream)
        for _ in range(args.steps):
            plain_step()
        e1.record(stream)
        e1.synchronize()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    ms = max_over_ranks(ws, ms)
    per_step = ms / args.steps
    flops = 2.0 * M * N * K
    value = ws * flops / (per_step * 1e-3) / 1e9
    launches = args.steps * 1

    # e2e through the drop-in (host-pointer) symbol with pinned host buffers
    hA = torch.from_numpy(A).pin_memory()
    hB = torch.from_numpy(B).pin_memory()
    hC = torch.empty(2 * M * N, dtype=torch.float64).pin_memory()
    e2e_steps = max(1, min(args.steps, 3))
    L.matmuldd_mm(hA.data_ptr(), hB.data_ptr(), hC.data_ptr(), M, K, N, RI)
    _lib.check_last("matmuldd_mm")
    barrier(ws)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        L.matmuldd_mm(hA.data_ptr(), hB.data_ptr(), hC.data_ptr(), M, K, N, RI)
    t_e2e = (time.perf_counter() - t0) / e2e_steps
    t_e2e = max_over_ranks(ws, t_e2e)
    _lib.check_last("matmuldd_mm")

    # roofline of the (plain) GEMM kernel on the FP64 pipe
    achieved = FP64_INSTR_PER_MAC * M * N * K / (per_step * 1e-3)
    roof = {"bound": "fp64", "achieved": achieved / 1e12, "peak": fp64_peak_instr / 1e12,
            "unit": "T FP64-instr/s", "frac": achieved / fp64_peak_instr, "traffic": None,
            "peak_source": "own FP64 FMA probe (multifloats_b200/csrc/peaks.cu), same process"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "DD-GFLOP/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded; hi = +-u 2^e, u~U[1,2), e~U{-16..16} per row of A / column of B)",
            "config": {"workload": "dd_gemm_4096_plain", "M": M, "N": N, "K": K,
                       "renorm_interval": RI, "form": "plain FP64 compensated (split-INT8 pending)",
                       "l2": "operands 256 MiB each > 126 MB L2, no flush needed",
                       "parallelism": f"replicas x{ws}"},
            "e2e": {"value": ws * flops / t_e2e / 1e9, "unit": "DD-GFLOP/s",
                    "h2d_bytes_per_step": int(A.nbytes + B.nbytes), "d2h_bytes_per_step": int(hC.numel() * 8)},
            "gpu_launches": launches,
            "roofline": roof,
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)


def run_reference(args, ws, rank):
    if rank != 0:
        return
    threads = cpu_threads()
    steps_total = args.steps + args.warmup
    target = min(20.0, max(2.0, args.ref_budget / max(1, steps_total)))
    kind, nb, fn = cpu_gemm_sample(target, threads)
    for _ in range(args.warmup):
        fn()
    times = [fn() for _ in range(args.steps)]
    dt = sum(times) / len(times)
    value = 2.0 * M * K * nb / dt / 1e9
    sample = (f"matmuldd_mm on A 4096x4096 times B 4096x{nb} (a column block of the 4096^3 "
              f"workload), ri={RI}, {threads} threads")
    line = {
        "metric": METRIC, "value": value, "unit": "DD-GFLOP/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": {"workload": "dd_gemm_4096", "M": M, "N": N, "K": K, "renorm_interval": RI},
        "cpu_baseline": {"value": value, "unit": "DD-GFLOP/s", "cores": threads, "kind": kind,
                         "sample": sample},
        "e2e": {"value": value, "unit": "DD-GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--ref-budget", type=float, default=120.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        # CPU-only arm: rank 0 measures, the other ranks exit without work
        run_reference(args, int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")))
        return
    ws, rank, local = dist_init()
    try:
        run_ours(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
