"""Small, self-ending workloads for profiling each hot kernel once under ncu.

    python -m multifloats_b200.profile_cases {split,plain,elementwise,reduce,all} [--n N]

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
    ap.add_argument("case", choices=["split", "plain", "elementwise", "reduce", "all"])
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
    torch.cuda.synchronize()
    print("ok")
    return 0


if __name__ == "__main__":
    sys.exit(main())
