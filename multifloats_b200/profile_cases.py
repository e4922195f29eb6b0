"""Small, self-ending workloads for profiling each hot kernel once under ncu.

    python -m multifloats_b200.profile_cases {split,crt,plain,elementwise,reduce,batched,gemv,blas,all} [--n N]

Inputs exceed the 126 MB L2 where DRAM figures matter, while the whole case
stays within a few GB of device memory and a few kernel launches.
"""
from __future__ import annotations

import argparse
import ctypes as C
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def main() -> int:
    import torch

    from multifloats_b200 import _lib, api
    from multifloats_b200 import workloads as W

    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["split", "crt", "plain", "elementwise", "reduce", "batched", "gemv", "blas",
                                     "all"])
    ap.add_argument("--n", type=int, default=2048, help="matrix size for split / plain")
    args = ap.parse_args()
    dev = torch.device("cuda:0")
    L = _lib.lib()
    sp = C.c_void_p(torch.cuda.current_stream().cuda_stream)

    def d(x):
        return torch.from_numpy(x).to(dev)

    if args.case in ("split", "all"):
        m = args.n
        a = d(W.dd_rowcol_scaled(m, m, 16, "row", 1))
        b = d(W.dd_rowcol_scaled(m, m, 16, "col", 2))
        c = torch.empty_like(a)
        _lib.check(L.mfcuda_matmuldd_mm_split(a.data_ptr(), b.data_ptr(), c.data_ptr(), m, m, m, 0, 8.0,
                                              None, 0, None, sp), "split")
    if args.case in ("crt", "all"):
        m = args.n
        a = d(W.dd_rowcol_scaled(m, m, 16, "row", 1))
        b = d(W.dd_rowcol_scaled(m, m, 16, "col", 2))
        c = torch.empty_like(a)
        _lib.check(L.mfcuda_matmuldd_mm_crt(a.data_ptr(), b.data_ptr(), c.data_ptr(), m, m, m, 0, 8.0,
                                            None, 0, None, sp), "crt")
    if args.case in ("plain", "all"):
        m = args.n
        a, b = d(W.dd_uniform(m * m, 1)), d(W.dd_uniform(m * m, 2))
        api.matmuldd_mm(a, b, m, m, m, 8)
    if args.case in ("elementwise", "all"):
        n = 1 << 24
        for op in ("exp", "log", "sin", "cos", "sqrt"):
            x = d(W.ELEMENTWISE_INPUTS[op](n, 3))
            api.unary(op, x)
            del x
    if args.case in ("reduce", "all"):
        n = 1 << 24
        x, y = d(W.dd_uniform(n, 4)), d(W.dd_uniform(n, 5))
        api.dot_product(x, y)
        api.sum_dd(x)
        api.norm2(x)
    if args.case in ("gemv", "all"):
        m = 4096
        a, x = d(W.dd_uniform(m * m, 8)), d(W.dd_uniform(m, 9))
        api.matmuldd_mv(a, x, m, m, 8)
        api.matmuldd_vm(x, a, m, m, 8)
    if args.case in ("blas", "all"):
        # wgemm in both accumulation forms and the blocked / chain wtrsm, n = 1024
        m = 1024
        a, b, c = d(W.dd_uniform(m * m, 10)), d(W.dd_uniform(m * m, 11)), d(W.dd_uniform(m * m, 12))
        api.wgemm("N", "N", m, m, m, (1.5, 0.0), a, m, b, m, (0.5, 0.0), c, m)
        api.wgemm("T", "N", m, m, m, (1.5, 0.0), a, m, b, m, (0.5, 0.0), c, m)
        t = d(W.dd_triangular(m, m, 13))
        api.wtrsm("L", "L", "N", "N", m, m, (1.0, 0.0), t, m, c, m)
        api.wtrsm("L", "L", "T", "N", m, m, (1.0, 0.0), t, m, c, m)
    if args.case == "batched":
        # the batched configuration: 2000 GEMMs, M, N, K log-uniform in [16, 1024],
        # plain and split plans (built-in tile choice), each run once
        import numpy as np

        rng = np.random.default_rng(2024)
        shapes = [tuple(int(v) for v in s) for s in np.exp(rng.uniform(np.log(16), np.log(1024), (2000, 3)))]
        tot = sum(m * k + k * n for m, k, n in shapes)
        buf = d(W.dd_uniform(tot, 7))
        out = torch.empty(2 * sum(m * n for m, _, n in shapes), dtype=torch.float64, device=dev)
        descs = (_lib.gemm_desc * len(shapes))()
        off = oc = 0
        for i, (m, k, n) in enumerate(shapes):
            descs[i].a = buf[2 * off:].data_ptr()
            off += m * k
            descs[i].b = buf[2 * off:].data_ptr()
            off += k * n
            descs[i].c = out[2 * oc:].data_ptr()
            oc += m * n
            descs[i].m, descs[i].k, descs[i].n = m, k, n
        for form in (0, 1):
            p = C.c_void_p()
            _lib.check(L.mfcuda_batch_create_gemm(descs, len(shapes), form, 8, 0, 8.0, 0, C.byref(p)), "batch")
            _lib.check(L.mfcuda_batch_run(p, sp), "run")
            _lib.check(L.mfcuda_batch_status(p), "status")
            L.mfcuda_batch_destroy(p)
    torch.cuda.synchronize()
    print("ok")
    return 0


if __name__ == "__main__":
    sys.exit(main())
