#!/usr/bin/env python3
"""Benchmark of the DD GEMM hot path on B200: DD-GFLOP/s at M=N=K=4096.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload X] [--no-configs] [--no-sharded] [--no-cpu-baseline]

One step = one C = A*B of 4096^3 real64x2 operands resident in HBM in the
split-INT8 form (CRT variant, tcgen05 tensor cores; each operand is 256 MiB,
larger than the 126 MB L2, so no flush is needed between steps).  DD-GFLOP/s =
2*M*N*K / seconds / 1e9.  The digit-sliced split form and the plain FP64
compensated kernel are timed on the same operands and reported beside it,
with the error of every output of the split result (on the device, against
the plain product) and of sampled outputs against the exact product, and
rows / columns of the plain result checked bit for bit.  With N GPUs (one
process per GPU under torchrun) every rank multiplies its own independent pair
of matrices (weak scaling, no collective on the data path); the timed region
is bracketed by a barrier and a device synchronise, and the time is the max
over ranks.  Rank 0 prints one JSON line.

Sub-records of the same line: `sharded` (every N: one 8192^3 CRT product in
column panels over the ranks and a 2^26 dot product over shards, through the
library's NCCL entry points, strong scaling), and at N = 1 `configs`: the other
configurations of the path (256^3 plain; the 2^26 elementwise maps and
reductions; 4096^3 / 8192^3 split forms for several exponent spreads; the
2000-problem batch and 10^4 ragged arrays; complex 4096^3, the 512-problem
complex batch), each with its times, roofline fraction and a parity verdict
on its own outputs.  `--workload X` prints one configuration as its own line.

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


def _measured_hbm() -> float:
    """Measured HBM copy bandwidth of this pool's B200s (GB/s), from
    MEASURED_PEAKS.json when present, else the earlier pool measurement."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"])
    except Exception:
        return 6650.0


HBM_GBS = _measured_hbm()


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
def gpu_uuid() -> str | None:
    try:
        import torch

        u = torch.cuda.get_device_properties(torch.cuda.current_device()).uuid
        return "GPU-" + str(u)
    except Exception:
        return None


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
class NvmlClocks:
    """Polls SM clock, power and clock-event reasons through NVML every 10 ms
    while active (read-only queries)."""

    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, uuid: str | None):
        self.samples = []
        self.handle = None
        self.maxclk = None
        try:
            import pynvml as N

            N.nvmlInit()
            self.N = N
            self.handle = N.nvmlDeviceGetHandleByUUID(uuid) if uuid else N.nvmlDeviceGetHandleByIndex(0)
            self.maxclk = N.nvmlDeviceGetMaxClockInfo(self.handle, N.NVML_CLOCK_SM)
        except Exception:
            self.handle = None

    def __enter__(self):
        self.stop = threading.Event()
        if self.handle is not None:
            self.th = threading.Thread(target=self._run, daemon=True)
            self.th.start()
        return self

    def _run(self):
        N = self.N
        get_reasons = getattr(N, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            N.nvmlDeviceGetCurrentClocksThrottleReasons
        while not self.stop.is_set():
            try:
                clk = N.nvmlDeviceGetClockInfo(self.handle, N.NVML_CLOCK_SM)
                rs = get_reasons(self.handle)
                pw = N.nvmlDeviceGetPowerUsage(self.handle) / 1000.0
                self.samples.append((clk, rs, pw))
            except Exception:
                pass
            time.sleep(0.01)

    def __exit__(self, *exc):
        self.stop.set()
        if self.handle is not None:
            self.th.join(timeout=2)

    def summary(self) -> dict:
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.maxclk, "reasons": [], "samples": 0}
        reasons = set()
        for _, rs, _ in self.samples:
            for bit, nm in self.REASONS.items():
                if rs & bit:
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(c for c, _, _ in self.samples), "sm_max_mhz": self.maxclk,
                "reasons": sorted(reasons), "samples": len(self.samples),
                "power_w_max": max(p for _, _, p in self.samples), "source": "NVML, 10 ms polling"}


def load_peaks_lib():
    p = C.CDLL(os.path.join(ROOT, "multifloats_b200", "libmfcuda_peaks.so"))
    p.mfpeak_fp64.argtypes = [C.c_int64, C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    p.mfpeak_int8.argtypes = [C.c_int, C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    return p


def int8_peaks(pk, sp, seconds: float = 1.5):
    """(burst, sustained, clocks) INT8 tensor throughput in ops/s: one probe
    launch after the warm-up, then probe launches back to back for `seconds`
    with the median over the second half and the NVML clocks seen there."""
    ms, ops = C.c_double(), C.c_double()
    if pk.mfpeak_int8(20000, sp, C.byref(ms), C.byref(ops)) != 0:
        return None, None, None
    burst = ops.value / (ms.value * 1e-3)
    rates = []
    t0 = time.perf_counter()
    with NvmlClocks(gpu_uuid()) as clk:
        while time.perf_counter() - t0 < seconds:
            if pk.mfpeak_int8(20000, sp, C.byref(ms), C.byref(ops)) != 0:
                return burst, None, None
            rates.append(ops.value / (ms.value * 1e-3))
    late = rates[len(rates) // 2:]
    return burst, statistics.median(late) if late else None, clk.summary()


def profile_traffic(kernel: str, workload: str):
    """DRAM bytes (read + write) per launch of `kernel` on `workload` from the
    committed ncu summary profiles/traffic_per_launch.txt, or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic_per_launch.txt")) as f:
            for line in f:
                parts = line.split()
                if len(parts) >= 3 and not line.startswith("#") and parts[0] == kernel and parts[1] == workload:
                    return int(parts[2])
    except OSError:
        pass
    return None


def run_ours(args, ws, rank, local):
    import torch

    from multifloats_b200 import _lib, accuracy
    from multifloats_b200 import workloads as W

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    L = _lib.lib()
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)

    # cpu baseline first (rank 0, N = 1 only) so it never overlaps GPU timing:
    # all host cores, and one thread beside it
    cpu = cpu1 = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        threads = cpu_threads()
        kind, nb, fn = cpu_gemm_sample(args.cpu_seconds, threads)
        dt = fn()
        cpu = {"value": 2.0 * M * K * nb / dt / 1e9, "unit": "DD-GFLOP/s", "cores": threads,
               "kind": kind,
               "sample": f"matmuldd_mm on A 4096x4096 times B 4096x{nb} (columns of the 4096^3 "
                         f"workload), ri={RI}, {threads} threads, {dt:.1f} s"}
        kind1, nb1, fn1 = cpu_gemm_sample(args.cpu_seconds / 3, 1)
        dt1 = fn1()
        cpu1 = {"value": 2.0 * M * K * nb1 / dt1 / 1e9, "unit": "DD-GFLOP/s", "cores": 1, "kind": kind1,
                "sample": f"matmuldd_mm on A 4096x4096 times B 4096x{nb1}, ri={RI}, 1 thread, {dt1:.1f} s"}
        log("cpu baseline:", cpu, cpu1)

    # split config: hi = +-u 2^e, u ~ U[1,2), e ~ U{-R..R} per row of A / column of B, R = 16
    R = 16
    A = W.dd_rowcol_scaled(M, K, R, "row", seed=10 + rank)
    B = W.dd_rowcol_scaled(K, N, R, "col", seed=20 + rank)
    dA = torch.from_numpy(A).to(dev)
    dB = torch.from_numpy(B).to(dev)
    dC = torch.empty(2 * M * N, dtype=torch.float64, device=dev)
    wsb = L.mfcuda_split_workspace_size(M, K, N)
    wcb = L.mfcuda_crt_workspace_size(M, K, N, 0)
    dWS = torch.empty(max(wsb, wcb), dtype=torch.uint8, device=dev)
    info = (C.c_int * 3)()
    _lib.check(L.mfcuda_matmuldd_mm_split(dA.data_ptr(), dB.data_ptr(), dC.data_ptr(), M, K, N, 0, 8.0,
                                          dWS.data_ptr(), wsb, info, sp), "split (info)")
    S, rho_a, rho_b = tuple(info)
    cinfo = (C.c_int * 4)()
    _lib.check(L.mfcuda_matmuldd_mm_crt(dA.data_ptr(), dB.data_ptr(), dC.data_ptr(), M, K, N, 0, 8.0,
                                        dWS.data_ptr(), wcb, cinfo, sp), "crt (info)")
    NMOD, _, _, WBITS = tuple(cinfo)

    def split_step():
        _lib.check(L.mfcuda_matmuldd_mm_split(dA.data_ptr(), dB.data_ptr(), dC.data_ptr(), M, K, N, 0, 8.0,
                                              dWS.data_ptr(), wsb, None, sp), "split")

    def crt_step():
        _lib.check(L.mfcuda_matmuldd_mm_crt(dA.data_ptr(), dB.data_ptr(), dC.data_ptr(), M, K, N, 0, 8.0,
                                            dWS.data_ptr(), wcb, None, sp), "crt")

    def plain_step(out):
        _lib.check(L.mfcuda_matmuldd_mm(dA.data_ptr(), dB.data_ptr(), out.data_ptr(), M, K, N, RI, sp),
                   "mfcuda_matmuldd_mm")

    def timed(step, nclk):
        """K steps after W warm-up steps (and more untimed steps until the GPU
        has run the form for 0.5 s: clocks settled), barrier + synchronize on
        both sides; per-phase times from the library's own events."""
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        while time.perf_counter() - t0 < 0.5:
            for _ in range(10):
                step()
            torch.cuda.synchronize()
        barrier(ws)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with NvmlClocks(gpu_uuid()) as clk:
            torch.cuda.synchronize()
            barrier(ws)
            L.mfcuda_phase_profile_begin()
            e0.record(stream)
            for _ in range(args.steps):
                step()
            e1.record(stream)
            e1.synchronize()
        sums = (C.c_double * 4)()
        ncalls = C.c_int64()
        _lib.check(L.mfcuda_phase_profile_end(sums, C.byref(ncalls)), "phase profile")
        torch.cuda.synchronize()
        ms = max_over_ranks(ws, e0.elapsed_time(e1))
        phase = {nm: sums[q] / max(1, ncalls.value) for q, nm in enumerate(["scan", "slice", "mma", "combine"])}
        nclk.append(clk.summary())
        return ms / args.steps, phase

    flops = 2.0 * M * N * K
    clks = []
    # the digit-sliced form first, then the CRT form (the headline: same operands,
    # same error target, fewer tensor-core products)
    split_ms, split_phase = timed(split_step, clks)
    per_step, phase = timed(crt_step, clks)
    value = ws * flops / (per_step * 1e-3) / 1e9
    split_val = ws * flops / (split_ms * 1e-3) / 1e9
    launches = 9 * args.steps  # init x2, scan x2, plan, slice x2, tcgen05 MMA, reconstruction

    # roofline denominators, measured in-process after the split forms' timed
    # regions (the sustained INT8 loop runs the GPU at its power cap)
    pk = load_peaks_lib()
    ms_p, ins_p = C.c_double(), C.c_double()
    pk.mfpeak_fp64(200000, sp, C.byref(ms_p), C.byref(ins_p))
    fp64_peak = ins_p.value / (ms_p.value * 1e-3)
    int8_burst, int8_sustained, int8_clk = int8_peaks(pk, sp)

    # ---- plain FP64 form on the same operands (its own output buffer) ----
    dCp = torch.empty_like(dC)
    plain_steps = max(1, min(args.steps, 3))
    plain_step(dCp)
    torch.cuda.synchronize()
    barrier(ws)
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with NvmlClocks(gpu_uuid()) as pclk:
        p0.record(stream)
        for _ in range(plain_steps):
            plain_step(dCp)
        p1.record(stream)
        p1.synchronize()
    plain_ms = max_over_ranks(ws, p0.elapsed_time(p1)) / plain_steps
    plain_val = ws * flops / (plain_ms * 1e-3) / 1e9
    plain_fp64 = FP64_INSTR_PER_MAC * M * N * K / (plain_ms * 1e-3)

    # accuracy of the CRT result just computed: every output against the plain
    # product on the device, and sampled outputs against the exact product
    acc = plain_parity = None
    if rank == 0:
        from oracle import oracle as O

        full = accuracy.full_error_real(dA, dB, dC, M, K, N, RI)
        Ch = dC.cpu().numpy()
        rng = np.random.default_rng(123)
        ii, jj = rng.integers(0, M, 256), rng.integers(0, N, 256)
        err, ab = O.gemm_errors(A, B, Ch, M, K, N, ii, jj)
        acc = {"error_every_output": full,
               "max_err_over_k_ulp_absab": float(np.max(np.abs(err) / (K * 2.0 ** -104 * ab))),
               "max_err_over_ulp_absab": float(np.max(np.abs(err) / (2.0 ** -104 * ab))),
               "apriori_bound_k_ulp": L.mfcuda_crt_bound(WBITS, rho_a, rho_b, K),
               "digit_sliced_apriori_bound_k_ulp": (S + 1) * 2.0 ** (106 - 8 * S + rho_a + rho_b),
               "samples": 256, "oracle": "exact superaccumulator (oracle/mf_oracle.c)",
               "ulp": "1 DD ulp = 2^-104",
               "note": "true error of every output <= error_every_output + 1 (plain product within 1 of exact)"}
        del Ch
        # the plain product: whole rows and columns bit-identical to the reference MAC order
        Cp = dCp.cpu().numpy().reshape(N, M, 2)
        rows, cols = [0, 1111, 2222, 4095], [0, 1357, 2468, 4095]
        ok_r = O.same_bits(np.stack([Cp[:, i, :] for i in rows]), O.matmul_mm_rows(A, B, M, K, N, RI, rows))
        ok_c = O.same_bits(Cp[cols], O.matmul_mm_columns(A, B, M, K, N, RI, cols))
        plain_parity = {"bit_exact": bool(ok_r.all() and ok_c.all()), "rows": rows, "columns": cols,
                        "against": "oracle (reference MAC order, src/float64x2/matmul.inc:6-39)"}
        del Cp
    del dCp

    # ---- e2e: the drop-in host-pointer symbol with pinned host buffers ----
    hA = torch.from_numpy(A).pin_memory()
    hB = torch.from_numpy(B).pin_memory()
    hC = torch.empty(2 * M * N, dtype=torch.float64).pin_memory()
    bound = C.c_double()
    L.matmuldd_mm_crt(hA.data_ptr(), hB.data_ptr(), hC.data_ptr(), M, K, N, 0, C.byref(bound))
    _lib.check_last("matmuldd_mm_crt")
    e2e_steps = max(1, min(args.steps, 5))
    barrier(ws)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        L.matmuldd_mm_crt(hA.data_ptr(), hB.data_ptr(), hC.data_ptr(), M, K, N, 0, C.byref(bound))
    t_e2e = max_over_ranks(ws, (time.perf_counter() - t0) / e2e_steps)
    _lib.check_last("matmuldd_mm_crt")
    del hA, hB, hC

    # roofline of the dominant kernel: split_mma_pair_kernel (CRT items: one
    # residue product per modulus) on the INT8 tensor pipe.  The CRT timed
    # region is K short steps (well under a second), so the burst figure of the
    # probe is the denominator; the sustained figure is given beside it.
    int8_ops = NMOD * 2.0 * M * N * K  # algorithmic INT8 ops per launch
    achieved = int8_ops / (phase["mma"] * 1e-3)
    split_achieved = (S * (S + 1) // 2) * 2.0 * M * N * K / (split_phase["mma"] * 1e-3)
    roof = {"bound": "tensor", "achieved": achieved / 1e12,
            "peak": int8_burst / 1e12 if int8_burst else None, "unit": "TFLOP/s",
            "frac": achieved / int8_burst if int8_burst else None,
            "traffic": profile_traffic("split_mma_pair_kernel", "dd_gemm_4096_crt"),
            "kernel": "split_mma_pair_kernel (CRT items)",
            "op_kind": "INT8 tensor ops (multiply + add), one residue product per modulus",
            "peak_source": "own tcgen05 kind::i8 probe (multifloats_b200/csrc/peaks.cu), same process, burst "
                           "(one probe launch; the timed region is short); of measured",
            "peak_sustained": int8_sustained / 1e12 if int8_sustained else None,
            "frac_of_sustained": achieved / int8_sustained if int8_sustained else None,
            "peak_sustained_clocks": int8_clk,
            "algorithmic_bytes": {"residues_read": 2 * NMOD * M * K, "residue_bytes_written": NMOD * M * N}}
    del dA, dB, dC, dWS
    torch.cuda.empty_cache()

    sharded = None
    if not args.no_sharded:
        sharded = measure_sharded(max(3, min(args.steps, 10)), args.warmup, ws, rank, dev, stream)

    configs = None
    if rank == 0 and ws == 1 and not args.no_configs:
        t0 = time.perf_counter()
        st, wu = max(3, min(args.steps, 10)), args.warmup
        configs = {"c1_gemm_256": measure_plain_256(),
                   "c2_elementwise_2^26": measure_elementwise(st, wu),
                   "c2_reductions_2^26_and_c5_complex_2^24": measure_reductions(st, wu),
                   "c3_split_4096_8192": measure_split_configs(max(3, st // 2), wu),
                   "c4_batched": measure_batched(max(3, st // 3), wu),
                   "c5_complex": measure_complex(max(3, st // 3), wu, reductions=False)}
        configs["parity_ok"] = all(v.get("parity_ok", all(r.get("parity_ok", True) for r in v.values()
                                                          if isinstance(r, dict)))
                                   for v in configs.values() if isinstance(v, dict))
        configs["seconds"] = time.perf_counter() - t0
        configs["clocks"] = _clock_summary()

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "DD-GFLOP/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int8+f64",
            "data": "synthetic (seeded; hi = +-u 2^e, u~U[1,2), e~U{-16..16} per row of A / column of B)",
            "config": {"workload": "dd_gemm_4096_split_int8", "M": M, "N": N, "K": K, "R": R,
                       "form": "crt (modular split-INT8)", "moduli": NMOD, "bits": WBITS,
                       "rho_a": rho_a, "rho_b": rho_b, "target": "err <= 8 k 2^-104 (|A||B|)_ij",
                       "l2": "operands 256 MiB each > 126 MB L2, no flush needed",
                       "parallelism": f"independent problem per GPU x{ws}"},
            "digit_sliced": {"value": split_val, "unit": "DD-GFLOP/s", "ms_per_step": split_ms, "slices": S,
                             "phases_ms": split_phase,
                             "mma_int8_tops": split_achieved / 1e12,
                             "mma_frac": split_achieved / int8_burst if int8_burst else None},
            "plain": {"value": plain_val, "unit": "DD-GFLOP/s", "ms_per_step": plain_ms, "steps": plain_steps,
                      "renorm_interval": RI, "fp64_instr_per_s": plain_fp64, "fp64_peak": fp64_peak,
                      "frac": plain_fp64 / fp64_peak, "clocks": pclk.summary(), "parity": plain_parity},
            "speedup_split_vs_plain": value / plain_val,
            "speedup_crt_vs_digit_sliced": value / split_val,
            "accuracy": acc,
            "phases_ms": phase,
            "e2e": {"value": ws * flops / t_e2e / 1e9, "unit": "DD-GFLOP/s",
                    "h2d_bytes_per_step": int(A.nbytes + B.nbytes), "d2h_bytes_per_step": int(2 * M * N * 8),
                    "call": "matmuldd_mm_crt (host pointers, pinned)"},
            "gpu_launches": launches,
            "roofline": roof,
            "cpu_baseline": cpu,
            "cpu_baseline_1thread": cpu1,
            "clocks": clks[-1],
            "clocks_digit_sliced": clks[0],
            "sharded": sharded,
            "configs": configs,
        }
        print(json.dumps(line), flush=True)


# ------------------------------------------------------- secondary workloads
# The other configurations of the hot path.  Each measure_* returns a record
# (times, roofline fractions and a parity verdict on the same run's outputs);
# the default line carries them as sub-records under "configs", and
# `--workload X` prints one of them as its own line.
_CLOCKS = []  # NVML clock summaries of every timed region of a secondary workload


def _events_time(fn, steps, warmup, stream, min_warm_s=0.3):
    """Mean CUDA-event time of `steps` calls after `warmup` calls and, for
    short kernels, more untimed calls until the GPU has been busy for at least
    min_warm_s seconds (clocks ramped up before the first timed call).  The
    SM clock is sampled during the timed region."""
    import torch

    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < min_warm_s:
        for _ in range(max(1, warmup)):
            fn()
        torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with NvmlClocks(gpu_uuid()) as clk:
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        e1.synchronize()
    _CLOCKS.append(clk.summary())
    return e0.elapsed_time(e1) / steps


def _clock_summary(since: int = 0) -> dict | None:
    cl = _CLOCKS[since:]
    if not cl:
        return None
    sm = [c["sm_mhz"] for c in cl if c.get("sm_mhz")]
    return {"sm_mhz_min_median": min(sm) if sm else None, "sm_max_mhz": cl[0].get("sm_max_mhz"),
            "reasons": sorted({r for c in cl for r in c.get("reasons", [])}), "timed_regions": len(cl)}


def _renorm_dev(h, l):
    import torch

    s = h + l
    bb = s - h
    e = (h - (s - bb)) + (l - bb)
    return torch.stack([s, e], dim=1).reshape(-1)


def _dev_dd_uniform(n, seed, dev, lo=-1.0, hi=1.0):
    """Device-side DD uniform[lo, hi) with lo-limb hi*2^-53*U[-1,1) (then two_sum)."""
    import torch

    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    h = torch.empty(n, dtype=torch.float64, device=dev).uniform_(lo, hi, generator=g)
    l = h * 2.0 ** -53 * torch.empty(n, dtype=torch.float64, device=dev).uniform_(-1.0, 1.0, generator=g)
    return _renorm_dev(h, l)


def _dev_elementwise_inputs(op, n, seed, dev):
    """The elementwise config distributions generated on the device (same
    distributions as multifloats_b200.workloads, another random stream):
    exp hi ~ U[-700, 700]; log / sqrt hi = 2^U[-1000, 1000]; sin / cos
    hi ~ U[-1e6, 1e6] with 10% moved within 1e-12 of a multiple of pi/2;
    lo = hi 2^-53 U[-1, 1), then two_sum."""
    import torch

    g = torch.Generator(device=dev)
    g.manual_seed(seed)

    def u(lo, hi):
        return torch.empty(n, dtype=torch.float64, device=dev).uniform_(lo, hi, generator=g)

    if op == "exp":
        h = u(-700.0, 700.0)
    elif op in ("log", "sqrt"):
        h = torch.exp2(u(-1000.0, 1000.0))
    else:
        h = u(-1e6, 1e6)
        near = u(0.0, 1.0) < 0.10
        kmax = int(1e6 / (np.pi / 2))
        kk = torch.floor(u(-kmax, kmax + 1))
        h = torch.where(near, kk * (np.pi / 2) + u(-1e-12, 1e-12), h)
    return _renorm_dev(h, h * 2.0 ** -53 * u(-1.0, 1.0))


def _dev_rowcol_scaled(rows, cols, R, per, seed, dev):
    """Column-major rows x cols DD matrix on the device, hi = +-u 2^e with
    u ~ U[1,2) and e ~ U{-R..R} per row ('row') or per column ('col'), lo as
    elsewhere (the split config's distribution, generated identically on
    every rank from the seed)."""
    import torch

    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    u = torch.empty(cols, rows, dtype=torch.float64, device=dev).uniform_(1.0, 2.0, generator=g)
    u = torch.where(torch.rand(cols, rows, generator=g, device=dev) < 0.5, -u, u)
    ne = rows if per == "row" else cols
    e = torch.randint(-R, R + 1, (ne,), generator=g, device=dev).to(torch.float64)
    h = u * torch.exp2(e[None, :] if per == "row" else e[:, None])
    lo = h * 2.0 ** -53 * torch.empty_like(h).uniform_(-1.0, 1.0, generator=g)
    return _renorm_dev(h.reshape(-1), lo.reshape(-1))


def _fp64_peak(stream):
    pk = load_peaks_lib()
    ms_p, ins_p = C.c_double(), C.c_double()
    pk.mfpeak_fp64(200000, C.c_void_p(stream.cuda_stream), C.byref(ms_p), C.byref(ins_p))
    return ins_p.value / (ms_p.value * 1e-3)


# FP64 thread instructions (DADD + DMUL + DFMA) per element of the elementwise
# kernels on the config distributions, from ncu counters
# (profiles/unary_kernel_fp64_instructions_2^24.md)
FP64_PER_ELEM = {"exp": 323.0, "log": 316.0, "sin": 827.5, "cos": 827.5, "sqrt": 25.4}


def measure_elementwise(steps, warmup, parity=True, adjacent=False, cpu=False):
    """Config 2 elementwise: exp / log / sin / cos / sqrt over 2^26 elements of
    their distributions; parity = every element bit-identical to the oracle."""
    import torch

    from multifloats_b200 import api
    from multifloats_b200 import workloads as W
    from oracle import oracle as O

    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream()
    n = 1 << 26
    fp64_peak = _fp64_peak(stream)
    res, cpu_res = {}, {}
    threads = cpu_threads()
    for op in W.ELEMENTWISE_INPUTS:
        x = _dev_elementwise_inputs(op, n, 100 + len(res), dev)
        y = torch.empty_like(x)
        ms = _events_time(lambda: api.unary(op, x, out=y), steps, warmup, stream)
        r = {"ms": ms, "gelem_per_s": n / ms / 1e6, "hbm_gbs": 32.0 * n / ms / 1e6,
             "fp64_instr_per_s": FP64_PER_ELEM[op] * n / (ms * 1e-3)}
        r["frac_fp64"] = r["fp64_instr_per_s"] / fp64_peak
        r["frac_hbm"] = r["hbm_gbs"] / HBM_GBS
        if parity:
            xh, yh = x.cpu().numpy(), y.cpu().numpy()
            same = O.same_bits(yh, O.unary(op, xh, threads=0))
            r["parity"] = {"bit_exact": bool(same.all()), "elements_checked": int(same.size),
                           "mismatches": int((~same).sum()), "against": "oracle (C restatement, pinned)"}
        res[op] = r
        if cpu and O.ref_available():
            xs = x[: 2 << 21].cpu().numpy()
            t0 = time.perf_counter()
            O.ref_unary(op, xs, threads=threads)
            cpu_res[op] = {"gelem_per_s": (1 << 21) / (time.perf_counter() - t0) / 1e9, "kind": "reference",
                           "cores": threads}
        del x, y
    out = {"elements": n, "per_op": res, "fp64_peak": fp64_peak,
           "fp64_peak_source": "own FP64 FMA probe (multifloats_b200/csrc/peaks.cu), same process",
           "roofline": {"bound": "fp64 (exp/log/sin/cos), hbm (sqrt)", "kernel": "unary_kernel<exp>",
                        "achieved": res["exp"]["fp64_instr_per_s"] / 1e12, "peak": fp64_peak / 1e12,
                        "unit": "T FP64-instr/s", "frac": res["exp"]["frac_fp64"], "traffic": None,
                        "hbm_peak_gbs": HBM_GBS, "sqrt_frac_hbm": res["sqrt"]["frac_hbm"]}}
    if parity:
        out["parity_ok"] = all(r["parity"]["bit_exact"] for r in res.values())
    if cpu_res:
        out["cpu_baseline_per_op"] = cpu_res
    if adjacent:
        # exp2 / log2 / log10, fused sincos (one reduction for both outputs)
        # against separate sin + cos, and the complex exp
        extra = {}
        for op, gen in W.EXTRA_ELEMENTWISE_INPUTS.items():
            x = torch.from_numpy(gen(n, seed=1)).to(dev)
            y = torch.empty_like(x)
            ms = _events_time(lambda: api.unary(op, x, out=y), steps, warmup, stream)
            extra[op] = {"ms": ms, "gelem_per_s": n / ms / 1e6}
            del x, y
        x = _dev_elementwise_inputs("sin", n, 1, dev)
        sv, cv = torch.empty_like(x), torch.empty_like(x)
        ms = _events_time(lambda: api.sincos(x, sv, cv), steps, warmup, stream)
        extra["sincos"] = {"ms": ms, "gelem_per_s": n / ms / 1e6,
                           "vs_sin_plus_cos": (res["sin"]["ms"] + res["cos"]["ms"]) / ms}
        del x, sv, cv
        nz = n // 2
        z = torch.stack([_dev_elementwise_inputs("exp", nz, 3, dev).view(-1, 2),
                         _dev_elementwise_inputs("sin", nz, 4, dev).view(-1, 2)], dim=1).reshape(-1)
        w = torch.empty_like(z)
        ms = _events_time(lambda: api.cexp(z, out=w), steps, warmup, stream)
        extra["cexp_2^25"] = {"ms": ms, "gelem_per_s": nz / ms / 1e6}
        del z, w
        out["adjacent_functions"] = extra
    torch.cuda.empty_cache()
    return out


def _reduction_fns(L, x, y, n, nc, out, ws, wsb, sp):
    """Device-pointer reduction calls on preallocated output and workspace
    (no per-call allocation): {kind: (call, bytes per element, elements)}."""
    def chk(rc):
        if rc:
            raise RuntimeError(f"reduction failed: {rc}")

    X, Y, O, WS = x.data_ptr(), y.data_ptr(), out.data_ptr(), ws.data_ptr()
    return {
        "sum": (lambda: chk(L.mfcuda_sumdd(X, n, O, WS, wsb, sp)), 16, n),
        "dot": (lambda: chk(L.mfcuda_dotdd(X, Y, n, RI, O, WS, wsb, sp)), 32, n),
        "norm2": (lambda: chk(L.mfcuda_norm2dd(X, n, O, WS, wsb, sp)), 16, n),
        "csum": (lambda: chk(L.mfcuda_csumdd(X, nc, O, WS, wsb, sp)), 32, nc),
        "cdot": (lambda: chk(L.mfcuda_cdotdd(X, Y, nc, RI, O, WS, wsb, sp)), 64, nc),
        "cnorm2": (lambda: chk(L.mfcuda_cnorm2dd(X, nc, O, WS, wsb, sp)), 32, nc),
    }


def measure_reductions(steps, warmup, parity=True):
    """Config 2 reductions over 2^26 real64x2 elements and config 5's complex
    ones over 2^24 complex64x2 elements (the first 2^25 DD of the same
    arrays); parity = bit-identical to the restated blocked order."""
    import torch

    from multifloats_b200 import _lib
    from oracle import oracle as O

    L = _lib.lib()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)
    n = 1 << 26
    nc = 1 << 24
    x, y = _dev_dd_uniform(n, 1, dev), _dev_dd_uniform(n, 2, dev)
    out = torch.empty(4, dtype=torch.float64, device=dev)
    wsb = L.mfcuda_reduce_workspace_size(n)
    ws = torch.empty(wsb, dtype=torch.uint8, device=dev)
    xh = yh = None
    if parity:
        xh, yh = x.cpu().numpy(), y.cpu().numpy()
    res = {}
    for kind, (fn, bpe, cnt) in _reduction_fns(L, x, y, n, nc, out, ws, wsb, sp).items():
        ms = _events_time(fn, steps, warmup, stream)
        res[kind] = {"ms": ms, "gbs": bpe * cnt / ms / 1e6, "frac_hbm": bpe * cnt / ms / 1e6 / HBM_GBS,
                     "elements": cnt}
        if parity:
            got = out.cpu().numpy()[: 4 if kind in ("csum", "cdot") else 2]
            span = 4 * cnt if kind.startswith("c") else 2 * cnt
            want = O.reduce_blocked(kind, xh[:span], yh[:span] if "dot" in kind else None, RI)
            res[kind]["parity"] = {"bit_exact": bool(O.same_bits(got, want).all()),
                                   "against": "oracle restatement of the device's blocked order"}
    del x, y, ws
    torch.cuda.empty_cache()
    rec = {"per_kind": res,
           "roofline": {"bound": "hbm", "kernel": "reduce_stage1<dot>", "achieved": res["dot"]["gbs"],
                        "peak": HBM_GBS, "unit": "GB/s", "frac": res["dot"]["frac_hbm"], "traffic": None,
                        "peak_source": "MEASURED_PEAKS.json hbm_gbs"}}
    if parity:
        rec["parity_ok"] = all(r["parity"]["bit_exact"] for r in res.values())
    return rec


def _batch_descs(shapes, dev, seed, width=2):
    """Device operands of a batch in one buffer (width 2: real64x2, 4:
    complex64x2) and the descriptor array."""
    import torch

    from multifloats_b200 import _lib

    tot = sum(m * k + k * n for m, k, n in shapes)
    buf = _dev_dd_uniform(tot * width // 2, seed, dev)
    out = torch.empty(width * sum(m * n for m, _, n in shapes), dtype=torch.float64, device=dev)
    descs = (_lib.gemm_desc * len(shapes))()
    offs = []
    off = oc = 0
    for i, (m, k, n) in enumerate(shapes):
        descs[i].a = buf[width * off:].data_ptr()
        oa = off
        off += m * k
        descs[i].b = buf[width * off:].data_ptr()
        ob = off
        off += k * n
        descs[i].c = out[width * oc:].data_ptr()
        offs.append((oa, ob, oc))
        oc += m * n
        descs[i].m, descs[i].k, descs[i].n = m, k, n
    return descs, (buf, out), offs


def _batch_parity(form, shapes, buf_h, out_h, offs, sample, cplx=False):
    """Sampled problems of a batch against the oracle: plain = one column
    bit-identical to the reference MAC order, CRT = one row bit-identical to
    the CRT restatement (real batches; complex batches: the whole problem)."""
    from oracle import oracle as O

    w = 4 if cplx else 2

    def check(i):
        m, k, n = shapes[i]
        oa, ob, oc = offs[i]
        a = buf_h[w * oa: w * (oa + m * k)]
        b = buf_h[w * ob: w * (ob + k * n)]
        c = out_h[w * oc: w * (oc + m * n)]
        if cplx:
            want = O.cmatmul_mm(a, b, m, k, n, RI) if form == "plain" else O.crt_cgemm(a, b, m, k, n)[0]
            return bool(O.same_bits(c, want).all())
        c3 = c.reshape(n, m, 2)
        if form == "plain":
            j = (7 * i) % n
            return bool(O.same_bits(c3[j], O.matmul_mm_columns(a, b, m, k, n, RI, [j], threads=1)[0]).all())
        r = (5 * i) % m
        want, _ = O.crt_gemm(a, b, m, k, n, rows=(r, r + 1))
        return bool(O.same_bits(c3[:, r, :], want.reshape(n, 2)).all())

    ok = O.parallel_map(check, sample)
    return {"bit_exact": all(ok), "problems_checked": len(sample),
            "what": ("whole problems" if cplx else ("one column per problem" if form == "plain"
                                                    else "one row per problem")),
            "against": "oracle (reference MAC order / CRT restatement)"}


def measure_batched(steps, warmup, parity=True):
    """Config 4: 2000 GEMMs with M, N, K log-uniform in [16, 1024] as one
    grouped launch per form (a CUDA graph), and 10^4 ragged exp / log arrays
    with lengths log-uniform in [64, 2^20]."""
    import torch

    from multifloats_b200 import _lib
    from oracle import oracle as O

    L = _lib.lib()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)
    rng = np.random.default_rng(2024)
    shapes = [tuple(int(v) for v in s) for s in np.exp(rng.uniform(np.log(16), np.log(1024), (2000, 3)))]
    flops = sum(2.0 * m * k * n for m, k, n in shapes)
    descs, keep, offs = _batch_descs(shapes, dev, 7)
    buf_h = keep[0].cpu().numpy() if parity else None
    sample = list(range(0, len(shapes), 10))
    res = {}
    for form, name in ((0, "plain"), (1, "split"), (2, "crt")):
        p = C.c_void_p()
        t0 = time.perf_counter()
        _lib.check(L.mfcuda_batch_create_gemm(descs, len(shapes), form, RI, 0, 8.0, 1, C.byref(p)), "batch")
        t_create = time.perf_counter() - t0
        ms = _events_time(lambda: _lib.check(L.mfcuda_batch_run(p, sp), "run"), steps, warmup, stream)
        _lib.check(L.mfcuda_batch_status(p), "status")
        res[name] = {"ms": ms, "dd_gflops": flops / ms / 1e6, "work_items": L.mfcuda_batch_work_items(p),
                     "plan_create_s": t_create}
        if parity and name in ("plain", "crt"):
            res[name]["parity"] = _batch_parity(name, shapes, buf_h, keep[1].cpu().numpy(), offs, sample)
        L.mfcuda_batch_destroy(p)
    del keep, buf_h
    torch.cuda.empty_cache()
    # 10^4 ragged exp / log arrays, lengths log-uniform in [64, 2^20]
    lens = [int(v) for v in np.exp(rng.uniform(np.log(64), np.log(1 << 20), 10000))]
    tot = sum(lens)
    x = _dev_dd_uniform(tot, 9, dev, 0.5, 2.0)
    yv = torch.empty_like(x)
    offs_r = np.concatenate([[0], np.cumsum(lens)])
    X = (C.c_void_p * len(lens))(*[x[2 * int(o):].data_ptr() for o in offs_r[:-1]])
    Y = (C.c_void_p * len(lens))(*[yv[2 * int(o):].data_ptr() for o in offs_r[:-1]])
    N = (C.c_int64 * len(lens))(*lens)
    for op, code in (("exp", 0), ("log", 1)):
        p = C.c_void_p()
        _lib.check(L.mfcuda_batch_create_unary(code, X, Y, N, len(lens), C.byref(p)), "ragged")
        ms = _events_time(lambda: _lib.check(L.mfcuda_batch_run(p, sp), "run"), steps, warmup, stream)
        r = {"ms": ms, "arrays": len(lens), "elements": tot, "gelem_per_s": tot / ms / 1e6}
        if parity:
            picks = list(range(0, len(lens), 50))
            xs = {i: x[2 * int(offs_r[i]):2 * int(offs_r[i + 1])].cpu().numpy() for i in picks}
            ys = {i: yv[2 * int(offs_r[i]):2 * int(offs_r[i + 1])].cpu().numpy() for i in picks}
            ok = O.parallel_map(lambda i: bool(O.same_bits(ys[i], O.unary(op, xs[i])).all()), picks)
            r["parity"] = {"bit_exact": all(ok), "arrays_checked": len(picks), "what": "whole arrays"}
        res["ragged_" + op] = r
        L.mfcuda_batch_destroy(p)
    del x, yv
    torch.cuda.empty_cache()
    best = max(("split", "crt"), key=lambda f: res[f]["dd_gflops"])
    rec = {"problems": len(shapes), "dd_gflop_per_step": flops / 1e9, "per_form": res, "best_split_form": best,
           "speedup_split_vs_plain": res[best]["dd_gflops"] / res["plain"]["dd_gflops"],
           "launch": "one CUDA graph per batch (grouped persistent kernels); autotuned tiles"}
    if parity:
        rec["parity_ok"] = all(r["parity"]["bit_exact"] for r in res.values() if "parity" in r)
    return rec


def _crt_call(L, dA, dB, dC, m, k, n, ws, wsb, sp, cplx=False, info=None):
    from multifloats_b200 import _lib

    sym = L.mfcuda_cmatmuldd_mm_crt if cplx else L.mfcuda_matmuldd_mm_crt
    _lib.check(sym(dA.data_ptr(), dB.data_ptr(), dC.data_ptr(), m, k, n, 0, 8.0, ws.data_ptr(), wsb, info, sp),
               "crt")


def measure_split_configs(steps, warmup, cases=((4096, 0), (4096, 64), (8192, 16)), parity=True):
    """Config 3: the split forms at M = N = K in {4096, 8192}, R in {0, 16, 64}:
    CRT and digit-sliced times, and the error of EVERY output of the CRT
    product (against the plain product on the device, in units of
    k 2^-104 (|A||B|)_ij; the true error is at most that plus 1) with 128
    outputs checked against the exact product."""
    import torch

    from multifloats_b200 import _lib, accuracy
    from multifloats_b200 import workloads as W
    from oracle import oracle as O

    L = _lib.lib()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)
    res = {}
    for n, R in cases:
        A = W.dd_rowcol_scaled(n, n, R, "row", 31 + R)
        B = W.dd_rowcol_scaled(n, n, R, "col", 41 + R)
        dA, dB = torch.from_numpy(A).to(dev), torch.from_numpy(B).to(dev)
        dC = torch.empty_like(dA)
        wsb = L.mfcuda_split_workspace_size(n, n, n)
        ws = torch.empty(wsb, dtype=torch.uint8, device=dev)
        info = (C.c_int * 3)()
        _lib.check(L.mfcuda_matmuldd_mm_split(dA.data_ptr(), dB.data_ptr(), dC.data_ptr(), n, n, n, 0, 8.0,
                                              ws.data_ptr(), wsb, info, sp), "split")
        ms_s = _events_time(lambda: _lib.check(L.mfcuda_matmuldd_mm_split(
            dA.data_ptr(), dB.data_ptr(), dC.data_ptr(), n, n, n, 0, 8.0, ws.data_ptr(), wsb, None, sp), "split"),
            steps, warmup, stream)
        del ws
        torch.cuda.empty_cache()
        wcb = L.mfcuda_crt_workspace_size(n, n, n, 0)
        wsc = torch.empty(wcb, dtype=torch.uint8, device=dev)
        cinfo = (C.c_int * 4)()
        _crt_call(L, dA, dB, dC, n, n, n, wsc, wcb, sp, info=cinfo)
        ms_c = _events_time(lambda: _crt_call(L, dA, dB, dC, n, n, n, wsc, wcb, sp), steps, warmup, stream)
        del wsc
        r = {"crt": {"ms": ms_c, "dd_gflops": 2.0 * n ** 3 / ms_c / 1e6, "moduli": cinfo[0], "bits": cinfo[3],
                     "apriori_bound_k_ulp": L.mfcuda_crt_bound(cinfo[3], cinfo[1], cinfo[2], n)},
             "digit_sliced": {"ms": ms_s, "dd_gflops": 2.0 * n ** 3 / ms_s / 1e6, "slices": info[0]},
             "rho_a": cinfo[1], "rho_b": cinfo[2]}
        if parity:
            r["crt"]["error_every_output"] = accuracy.full_error_real(dA, dB, dC, n, n, n, RI)
            rng = np.random.default_rng(R + n)
            ii, jj = rng.integers(0, n, 128), rng.integers(0, n, 128)
            err, ab = O.gemm_errors(A, B, dC.cpu().numpy(), n, n, n, ii, jj)
            r["crt"]["error_sampled_exact"] = {
                "samples": 128, "max_err_over_k_ulp_absab": float(np.max(np.abs(err) / (n * 2.0 ** -104 * ab))),
                "oracle": "exact superaccumulator"}
            worst = r["crt"]["error_every_output"]["max_err_vs_plain_k_ulp_absab"]
            r["parity_ok"] = bool(worst is not None and worst + 1.0 <= 8.0 and
                                  r["crt"]["error_sampled_exact"]["max_err_over_k_ulp_absab"] <= 8.0)
        res[f"{n}_R{R}"] = r
        log(n, R, json.dumps(r))
        del dA, dB, dC
        torch.cuda.empty_cache()
    return res


def measure_complex(steps, warmup, parity=True, reductions=True):
    """Config 5: complex64x2 4096^3 in the CRT form (four real products), the
    digit-sliced and plain forms beside it, the error of every output; a batch
    of 512 complex GEMMs with M, N, K log-uniform in [32, 512]; and (with
    reductions) complex dot / norm2 over 2^24 elements."""
    import torch

    from multifloats_b200 import _lib, accuracy
    from multifloats_b200 import workloads as W

    L = _lib.lib()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)
    m = 4096
    A = torch.from_numpy(W.complex_from_parts(W.dd_rowcol_scaled(m, m, 16, "row", 1),
                                              W.dd_rowcol_scaled(m, m, 16, "row", 2))).to(dev)
    B = torch.from_numpy(W.complex_from_parts(W.dd_rowcol_scaled(m, m, 16, "col", 3),
                                              W.dd_rowcol_scaled(m, m, 16, "col", 4))).to(dev)
    Cm = torch.empty_like(A)
    wsb = L.mfcuda_csplit_workspace_size(m, m, m)
    ws = torch.empty(wsb, dtype=torch.uint8, device=dev)
    ms_s = _events_time(lambda: _lib.check(L.mfcuda_cmatmuldd_mm_split(
        A.data_ptr(), B.data_ptr(), Cm.data_ptr(), m, m, m, 0, 8.0, ws.data_ptr(), wsb, None, sp), "cs"),
        steps, warmup, stream)
    ms_p = _events_time(lambda: _lib.check(L.mfcuda_cmatmuldd_mm(
        A.data_ptr(), B.data_ptr(), Cm.data_ptr(), m, m, m, RI, sp), "cp"), 1, 1, stream)
    del ws
    torch.cuda.empty_cache()
    wcb = L.mfcuda_ccrt_workspace_size(m, m, m, 0)
    wsc = torch.empty(wcb, dtype=torch.uint8, device=dev)
    ms_c = _events_time(lambda: _crt_call(L, A, B, Cm, m, m, m, wsc, wcb, sp, cplx=True), steps, warmup, stream)
    del wsc
    torch.cuda.empty_cache()
    flops = 8.0 * m ** 3  # four real products
    rec = {"crt": {"ms": ms_c, "dd_gflops": flops / ms_c / 1e6},
           "digit_sliced": {"ms": ms_s, "dd_gflops": flops / ms_s / 1e6},
           "plain": {"ms": ms_p, "dd_gflops": flops / ms_p / 1e6},
           "speedup_crt_vs_plain": ms_p / ms_c, "speedup_crt_vs_digit_sliced": ms_s / ms_c,
           "flops": "8 m n k (four real products)"}
    if parity:
        rec["crt"]["error_every_output"] = accuracy.full_error_complex(A, B, Cm, m, m, m, RI)
        worst = rec["crt"]["error_every_output"]["max_err_vs_plain_k_ulp_absab"]
        rec["parity_ok"] = bool(worst is not None and worst + 1.0 <= 8.0)
    del A, B, Cm
    torch.cuda.empty_cache()
    # batch of 512 complex GEMMs, M, N, K log-uniform in [32, 512]: plain, split and CRT plans
    rng = np.random.default_rng(512)
    shapes = [tuple(int(v) for v in s_) for s_ in np.exp(rng.uniform(np.log(32), np.log(512), (512, 3)))]
    bflops = sum(8.0 * mm * kk * nn for mm, kk, nn in shapes)
    descs, keep, offs = _batch_descs(shapes, dev, 8, width=4)
    buf_h = keep[0].cpu().numpy() if parity else None
    batch = {}
    for form, name in ((0, "plain"), (1, "split"), (2, "crt")):
        p = C.c_void_p()
        _lib.check(L.mfcuda_batch_create_cgemm(descs, len(shapes), form, RI, 0, 8.0, 1, C.byref(p)), "cbatch")
        bms = _events_time(lambda: _lib.check(L.mfcuda_batch_run(p, sp), "run"), steps, warmup, stream)
        _lib.check(L.mfcuda_batch_status(p), "status")
        batch[name] = {"ms": bms, "dd_gflops": bflops / bms / 1e6, "work_items": L.mfcuda_batch_work_items(p)}
        if parity and name in ("plain", "crt"):  # whole problems up to 256^3 (CPU time)
            sample = [i for i in range(0, len(shapes), 8) if shapes[i][0] * shapes[i][1] * shapes[i][2] <= 1 << 24]
            batch[name]["parity"] = _batch_parity(name, shapes, buf_h, keep[1].cpu().numpy(), offs, sample,
                                                  cplx=True)
        L.mfcuda_batch_destroy(p)
    del keep, buf_h
    torch.cuda.empty_cache()
    rec["batch_512_complex_32_512"] = {**batch, "speedup_split_vs_plain": batch["plain"]["ms"] / batch["split"]["ms"],
                                       "speedup_crt_vs_plain": batch["plain"]["ms"] / batch["crt"]["ms"],
                                       "real_dd_gflop_per_step": bflops / 1e9}
    if parity:
        rec["parity_ok"] = rec.get("parity_ok", True) and all(
            b["parity"]["bit_exact"] for b in batch.values() if "parity" in b)
    if reductions:
        red = measure_reductions(steps, warmup, parity=parity)
        rec["cdot_2^24"] = red["per_kind"]["cdot"]
        rec["cnorm2_2^24"] = red["per_kind"]["cnorm2"]
    return rec


def measure_plain_256(parity=True):
    """Config 1: 256^3 plain compensated product, bit-identical to the
    reference MAC order in full."""
    import torch

    from multifloats_b200 import api
    from multifloats_b200 import workloads as W
    from oracle import oracle as O

    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream()
    m = 256
    a, b = W.dd_uniform(m * m, seed=0), W.dd_uniform(m * m, seed=1)
    da, db = torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)
    dc = torch.empty_like(da)
    ms = _events_time(lambda: api.matmuldd_mm(da, db, m, m, m, RI, out=dc), 20, 3, stream, min_warm_s=0.0)
    rec = {"ms": ms, "dd_gflops": 2.0 * m ** 3 / ms / 1e6}
    if parity:
        rec["parity"] = {"bit_exact": bool(O.same_bits(dc.cpu().numpy(), O.matmul_mm(a, b, m, m, m, RI)).all()),
                         "what": "every output", "against": "oracle (reference MAC order)"}
        rec["parity_ok"] = rec["parity"]["bit_exact"]
    return rec


def measure_sharded(steps, warmup, ws, rank, dev, stream):
    """The multi-GPU design through the C ABI (NCCL): one 8192^3 product in the
    CRT form split into column panels over the ranks (strong scaling; every
    rank holds A and B, computes its panel; the plan agreed by one on-stream
    MAX all-reduce), the same with every panel gathered on every rank, and a
    2^26 dot product over contiguous shards (all-gather of partials, rank-order
    fold).  Times are the max over ranks.  Parity (rank 0): the gathered C is
    bit-identical to the single-device call; the dot product is bit-identical
    to the oracle's rank-order fold of the shards' partials."""
    import torch

    from multifloats_b200 import _lib
    from multifloats_b200.nccl_comm import NcclComm

    L = _lib.lib()
    sp = C.c_void_p(stream.cuda_stream)
    comm = NcclComm.single(dev.index) if ws == 1 else NcclComm.from_process_group(rank, ws)
    rec = {"ranks": ws, "via": "mfcuda_matmuldd_mm_nccl / mfcuda_reduce_nccl (NCCL communicator of the ranks)"}
    try:
        n = 8192
        dA = _dev_rowcol_scaled(n, n, 16, "row", 501, dev)
        dB = _dev_rowcol_scaled(n, n, 16, "col", 502, dev)
        dC = torch.empty_like(dA)
        j0, j1 = C.c_int64(), C.c_int64()
        L.mfcuda_shard_bounds(n, rank, ws, C.byref(j0), C.byref(j1))
        wcb = L.mfcuda_crt_workspace_size(n, n, max(1, j1.value - j0.value), 0)
        wsp = torch.empty(wcb, dtype=torch.uint8, device=dev)

        def prod(flags):
            _lib.check(L.mfcuda_matmuldd_mm_nccl(2, dA.data_ptr(), dB.data_ptr(), dC.data_ptr(), n, n, n, 0, 8.0,
                                                 flags, wsp.data_ptr(), wcb, None, comm.handle, sp), "nccl crt")

        def timed(fn, k):
            for _ in range(warmup):
                fn()
            torch.cuda.synchronize()
            barrier(ws)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(k):
                fn()
            e1.record(stream)
            e1.synchronize()
            return max_over_ranks(ws, e0.elapsed_time(e1)) / k

        k = max(3, steps)
        ms = timed(lambda: prod(0), k)
        ms_g = timed(lambda: prod(2), k)
        rec["crt_8192_panels"] = {"ms": ms, "dd_gflops": 2.0 * n ** 3 / ms / 1e6,
                                  "panel_columns": [j0.value, j1.value]}
        rec["crt_8192_panels_gathered"] = {"ms": ms_g, "dd_gflops": 2.0 * n ** 3 / ms_g / 1e6}
        if rank == 0:  # dC holds all of C after the gathered call
            del wsp
            single = torch.empty_like(dC)
            wfull = L.mfcuda_crt_workspace_size(n, n, n, 0)
            wsf = torch.empty(wfull, dtype=torch.uint8, device=dev)
            _lib.check(L.mfcuda_matmuldd_mm_crt(dA.data_ptr(), dB.data_ptr(), single.data_ptr(), n, n, n, 0, 8.0,
                                                wsf.data_ptr(), wfull, None, sp), "single crt")
            torch.cuda.synchronize()
            same = bool(torch.equal(single.view(torch.int64), dC.view(torch.int64)))
            rec["crt_8192_panels_gathered"]["parity"] = {"bit_exact_vs_single_call": same}
            del single, wsf
        del dA, dB, dC
        torch.cuda.empty_cache()
        barrier(ws)
        # 2^26 dot product over contiguous shards
        nd = 1 << 26
        x, y = _dev_dd_uniform(nd, 601, dev), _dev_dd_uniform(nd, 602, dev)
        L.mfcuda_shard_bounds(nd, rank, ws, C.byref(j0), C.byref(j1))
        xs, ys = x[2 * j0.value:2 * j1.value], y[2 * j0.value:2 * j1.value]
        out = torch.empty(2, dtype=torch.float64, device=dev)
        nloc = j1.value - j0.value

        def dot():
            _lib.check(L.mfcuda_reduce_nccl(1, xs.data_ptr(), ys.data_ptr(), nloc, RI, out.data_ptr(), comm.handle,
                                            sp), "nccl dot")

        ms_d = timed(dot, max(10, steps))
        rec["dot_2^26"] = {"ms": ms_d, "gbs": 32.0 * nd / ms_d / 1e6}
        if rank == 0:
            from oracle import oracle as O

            xh, yh = x.cpu().numpy(), y.cpu().numpy()
            parts = []
            for r in range(ws):
                L.mfcuda_shard_bounds(nd, r, ws, C.byref(j0), C.byref(j1))
                parts.append(O.reduce_partial("dot", xh[2 * j0.value:2 * j1.value], yh[2 * j0.value:2 * j1.value],
                                              RI))
            want = O.reduce_combine("dot", np.concatenate(parts))
            rec["dot_2^26"]["parity"] = {
                "bit_exact_vs_rank_order_fold": bool(O.same_bits(out.cpu().numpy(), want).all())}
        del x, y
        torch.cuda.empty_cache()
    finally:
        torch.cuda.synchronize()
        barrier(ws)
        comm.close()
    if rank == 0:
        rec["parity_ok"] = bool(rec["crt_8192_panels_gathered"]["parity"]["bit_exact_vs_single_call"] and
                                rec["dot_2^26"]["parity"]["bit_exact_vs_rank_order_fold"])
    return rec


def _line(args, workload, metric, value, unit, extra):
    d = {"metric": metric, "value": value, "unit": unit, "n_gpus": 1, "steps": args.steps,
         "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
         "data": "synthetic (seeded)", "config": {"workload": workload}}
    d.update(extra)
    if _CLOCKS:
        d["clocks"] = _clock_summary()
    print(json.dumps(d), flush=True)


def run_elementwise(args):
    rec = measure_elementwise(args.steps, args.warmup, parity=True, adjacent=True, cpu=not args.no_cpu_baseline)
    _line(args, "dd_elementwise_2^26", "DD elementwise G elem/s, 2^26 elements (exp/log/sin/cos/sqrt)",
          rec["per_op"]["exp"]["gelem_per_s"], "G elem/s (exp)", {"dtype": "f64", **rec})


def run_reductions(args):
    rec = measure_reductions(args.steps, args.warmup, parity=True)
    _line(args, "dd_reductions_2^26", "DD reductions GB/s (dot 2^26)", rec["per_kind"]["dot"]["gbs"], "GB/s",
          {"dtype": "f64", **rec})


def run_batched(args):
    rec = measure_batched(max(1, args.steps // 3), args.warmup, parity=True)
    best = rec["best_split_form"]
    _line(args, "dd_batched_2000_gemms_16_1024",
          "Batched DD-GEMM DD-GFLOP/s, 2000 problems M,N,K log-uniform [16,1024]",
          rec["per_form"][best]["dd_gflops"], "DD-GFLOP/s", {"dtype": "int8+f64", **rec})


def run_complex(args):
    rec = measure_complex(max(1, args.steps // 3), args.warmup, parity=True)
    _line(args, "complex_dd_gemm_4096_split",
          "complex64x2 GEMM 4096^3 real DD-GFLOP/s (8mnk), split-INT8 (CRT form) vs plain",
          rec["crt"]["dd_gflops"], "DD-GFLOP/s", {"dtype": "int8+f64", **rec})


def run_gemm8192(args):
    res = measure_split_configs(max(1, args.steps // 5), args.warmup,
                                cases=((4096, 0), (4096, 16), (4096, 64), (8192, 0), (8192, 16), (8192, 64)))
    _line(args, "dd_gemm_split_4096_8192_R", "split-INT8 DD-GEMM DD-GFLOP/s 8192^3 (R=16), CRT form",
          res["8192_R16"]["crt"]["dd_gflops"], "DD-GFLOP/s",
          {"dtype": "int8+f64", "per_config": res, "ulp": "1 DD ulp = 2^-104"})


def run_gemv(args):
    """matmuldd_mv / matmuldd_vm device paths (HBM-bound: 16 bytes of the
    matrix per MAC), bit-identical to the reference's sequential MAC."""
    import torch

    from multifloats_b200 import _lib

    L = _lib.lib()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)
    res = {}
    for m in (4096, 16384):
        A = _dev_dd_uniform(m * m, 3, dev)
        x = _dev_dd_uniform(m, 4, dev)
        yv = torch.empty(2 * m, dtype=torch.float64, device=dev)

        def mv():
            _lib.check(L.mfcuda_matmuldd_mv(A.data_ptr(), x.data_ptr(), yv.data_ptr(), m, m, RI, sp), "mv")

        def vm():
            _lib.check(L.mfcuda_matmuldd_vm(x.data_ptr(), A.data_ptr(), yv.data_ptr(), m, m, RI, sp), "vm")

        for name, fn in (("mv", mv), ("vm", vm)):
            ms = _events_time(fn, args.steps, args.warmup, stream)
            gbs = 16.0 * m * m / ms / 1e6
            res[f"{name}_{m}"] = {"ms": ms, "gbs": gbs, "frac_hbm": gbs / HBM_GBS,
                                  "dd_gflops": 2.0 * m * m / ms / 1e6}
        del A, x, yv
        torch.cuda.empty_cache()
    _line(args, "dd_gemv_4096_16384", "DD matrix-vector GB/s (matrix bytes / time), mv 16384^2",
          res["mv_16384"]["gbs"], "GB/s",
          {"dtype": "f64", "per_case": res,
           "roofline": {"bound": "hbm", "kernel": "gemv_dd_kernel", "achieved": res["mv_16384"]["gbs"],
                        "peak": HBM_GBS, "unit": "GB/s", "frac": res["mv_16384"]["frac_hbm"], "traffic": None,
                        "peak_source": "MEASURED_PEAKS.json hbm_gbs"}})


def _dev_triangular(n, seed, dev):
    """n x n DD matrix, off-diagonal U[-1,1)/n, diagonal +-U[1,2) (diagonally
    dominant: repeated solves stay bounded)."""
    import torch

    a = _dev_dd_uniform(n * n, seed, dev).view(n, n, 2)
    a /= float(n)
    g = torch.Generator(device=dev)
    g.manual_seed(seed + 1)
    d = torch.empty(n, dtype=torch.float64, device=dev).uniform_(1.0, 2.0, generator=g)
    d *= torch.where(torch.rand(n, generator=g, device=dev) < 0.5, -1.0, 1.0)
    idx = torch.arange(n, device=dev)
    a[idx, idx, 0] = d
    a[idx, idx, 1] = 0.0
    return a.reshape(-1)


# FP64 instructions per wgemm / wtrsm multiply-add: DD multiply (two_prod 2, cross
# terms 4, fast_two_sum 3) + DD add or subtract (two two_sums 11 with the shared
# leading sum, 2 adds, 2 fast_two_sums 6 -> 20): 29 (the zero / non-finite tests
# are integer or predicate work).
BLAS_FP64_PER_MAC = 29.0


def run_blas(args):
    """BLAS-style shims (DGEMM / DTRSM semantics over DD matrices): wgemm at
    4096^3 in both accumulation forms and wtrsm 4096 x 4096 on the left and on
    the right; bit-identical to the reference shims' loops (tests)."""
    import torch

    from multifloats_b200 import api
    from multifloats_b200 import workloads as W
    from oracle import oracle as O

    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream()
    n = 4096
    A = _dev_dd_uniform(n * n, 11, dev)
    B = _dev_dd_uniform(n * n, 12, dev)
    Cm = _dev_dd_uniform(n * n, 13, dev)
    alpha, beta = np.array([1.5, 0.0]), np.array([0.5, 0.0])
    res = {}
    for ta, tb in (("N", "N"), ("T", "N"), ("N", "T")):
        ms = _events_time(lambda: api.wgemm(ta, tb, n, n, n, alpha, A, n, B, n, beta, Cm, n),
                          args.steps, args.warmup, stream, min_warm_s=0.0)
        res[f"wgemm_{ta}{tb}"] = {"ms": ms, "dd_gflops": 2.0 * n ** 3 / ms / 1e6,
                                  "fp64_instr_per_s": BLAS_FP64_PER_MAC * n ** 3 / (ms * 1e-3)}
    del A, B, Cm
    T = _dev_triangular(n, 21, dev)
    X = _dev_dd_uniform(n * n, 22, dev)
    one = np.array([1.0, 0.0])
    # six (side, uplo, trans) cases run the blocked right-looking solve; L-L-T and
    # R-L-N are one sequential chain per vector (their update order runs against
    # the pivot order), latency-bound
    for side, uplo, ta in (("L", "L", "N"), ("L", "U", "T"), ("R", "U", "N"), ("R", "L", "T"),
                           ("L", "L", "T"), ("R", "L", "N")):
        ms = _events_time(lambda: api.wtrsm(side, uplo, ta, "N", n, n, one, T, n, X, n),
                          args.steps, args.warmup, stream, min_warm_s=0.0)
        macs = n * n * (n - 1) / 2.0
        res[f"wtrsm_{side}{uplo}{ta}N"] = {"ms": ms, "dd_gflops": 2.0 * macs / ms / 1e6,
                                           "fp64_instr_per_s": BLAS_FP64_PER_MAC * macs / (ms * 1e-3)}
    del T, X
    torch.cuda.empty_cache()
    # end to end through the Fortran-callable host drop-in wgemm_ (host buffers,
    # copies inside the timed region)
    Ah, Bh = W.dd_uniform(n * n, seed=31), W.dd_uniform(n * n, seed=32)
    Ch = W.dd_uniform(n * n, seed=33)
    e2e_steps = max(1, min(args.steps, 3))
    api.wgemm("N", "N", n, n, n, alpha, Ah, n, Bh, n, beta, Ch, n)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        api.wgemm("N", "N", n, n, n, alpha, Ah, n, Bh, n, beta, Ch, n)
    e2e_ms = (time.perf_counter() - t0) * 1e3 / e2e_steps
    del Ah, Bh, Ch
    pk = load_peaks_lib()
    sp = C.c_void_p(stream.cuda_stream)
    ms_p, ins_p = C.c_double(), C.c_double()
    pk.mfpeak_fp64(200000, sp, C.byref(ms_p), C.byref(ins_p))
    fp64_peak = ins_p.value / (ms_p.value * 1e-3)
    for r in res.values():
        r["frac_fp64"] = r["fp64_instr_per_s"] / fp64_peak
    cpu = None
    if O.ref_available() and not args.no_cpu_baseline:
        threads = cpu_threads()
        s = 1024
        a, b, c = W.dd_uniform(s * s, seed=1), W.dd_uniform(s * s, seed=2), W.dd_uniform(s * s, seed=3)
        t0 = time.perf_counter()
        O.ref_wgemm("N", "N", s, s, s, alpha, a, s, b, s, beta, c, s, threads=threads)
        dt = time.perf_counter() - t0
        cpu = {"value": 2.0 * s ** 3 / dt / 1e9, "unit": "DD-GFLOP/s", "cores": threads, "kind": "reference",
               "sample": f"wgemm NN {s}^3 (the reference's DD operators in wgemm.f90's loop order, "
                         f"columns sharded over threads)"}
    head = res["wgemm_NN"]
    _line(args, "dd_wgemm_4096_wtrsm_4096", "DD BLAS-shim DD-GFLOP/s, wgemm NN 4096^3 (alpha, beta general)",
          head["dd_gflops"], "DD-GFLOP/s",
          {"dtype": "f64", "per_case": res, "cpu_baseline": cpu,
           "e2e": {"value": 2.0 * n ** 3 / e2e_ms / 1e6, "unit": "DD-GFLOP/s", "ms": e2e_ms,
                   "h2d_bytes_per_step": 3 * 16 * n * n, "d2h_bytes_per_step": 16 * n * n,
                   "path": "wgemm_ (Fortran-callable host drop-in)"},
           "roofline": {"bound": "fp64", "kernel": "wgemm_kernel<false,false,true>",
                        "achieved": head["fp64_instr_per_s"] / 1e12, "peak": fp64_peak / 1e12,
                        "unit": "T FP64-instr/s", "frac": head["frac_fp64"], "traffic": None,
                        "fp64_instr_per_mac": BLAS_FP64_PER_MAC,
                        "peak_source": "own FP64 FMA probe (multifloats_b200/csrc/peaks.cu), same process"}})


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
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded; hi = +-u 2^e, u~U[1,2), e~U{-16..16} per row of A / column of B)",
        "impl": "reference",
        "config": {"workload": "dd_gemm_4096_split_int8", "M": M, "N": N, "K": K, "R": 16,
                   "renorm_interval": RI, "parallelism": f"independent problem per GPU x{ws}",
                   "form": "the reference library's CPU matmuldd_mm (plain compensated form; the "
                           "reference has no split form), built from its sources, all host cores"},
        "cpu_baseline": {"value": value, "unit": "DD-GFLOP/s", "cores": threads, "kind": kind,
                         "sample": sample},
        "e2e": {"value": value, "unit": "DD-GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--ref-budget", type=float, default=120.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-sharded", action="store_true",
                    help="skip the NCCL column-panel / sharded-reduction sub-record")
    ap.add_argument("--no-configs", action="store_true",
                    help="headline only: skip the sub-records of the other configurations")
    ap.add_argument("--workload", default="gemm4096",
                    choices=["gemm4096", "elementwise", "reductions", "batched", "complex", "gemm8192", "gemv",
                             "blas"])
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        # CPU-only arm: rank 0 measures, the other ranks exit without work
        run_reference(args, int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")))
        return
    if args.workload != "gemm4096":
        {"elementwise": run_elementwise, "reductions": run_reductions, "batched": run_batched,
         "complex": run_complex, "gemm8192": run_gemm8192, "gemv": run_gemv,
         "blas": run_blas}[args.workload](args)
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
