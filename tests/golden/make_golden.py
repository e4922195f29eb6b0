"""Generate tests/golden/golden.npz from the reference library itself.

Run in a checkout where the reference sources were compiled into
oracle/_ref/libmfref.so (``make -C oracle``):

    python tests/golden/make_golden.py

Every output stored here was computed by the reference's own exported
functions (expdd, logdd, sindd, cosdd, sqrtdd, exp2dd, log2dd, log10dd,
sincosdd, cexpidd, cexpdd, adddd..divdd, matmuldd_mm/mv/vm)
or by compositions of them that mirror the Fortran layer (complex matmul from
four matmuldd_mm calls and the DD operators; norm2 from the DD operators and
sqrtdd).  Inputs are seeded and regenerable.  The fixtures let the tests pin
the oracle and the GPU kernels on machines where the reference is absent.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from multifloats_b200 import workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.npz")


def dd_list(values) -> np.ndarray:
    """(hi, lo) pairs -> interleaved array."""
    return np.array([[float(h), float(l)] for h, l in values], dtype=np.float64).reshape(-1)


def dd_from_mp(vals) -> np.ndarray:
    from mpmath import mp, mpf

    mp.prec = 300
    out = []
    for v in vals:
        v = mpf(v)
        hi = float(v)
        lo = float(v - mpf(hi))
        out.append((hi, lo))
    return dd_list(out)


def edge_inputs() -> dict[str, np.ndarray]:
    from mpmath import mp, mpf, pi, sqrt, e

    mp.prec = 300
    inf, nan = float("inf"), float("nan")
    tiny = 5e-324
    common = [
        (0.0, 0.0), (-0.0, 0.0), (0.0, -0.0), (-0.0, -0.0), (inf, 0.0), (-inf, 0.0), (nan, 0.0),
        (1.0, 0.0), (-1.0, 0.0), (2.0, 0.0), (0.5, 0.0), (3.0, 0.0), (tiny, 0.0), (-tiny, 0.0),
        (2.2250738585072014e-308, 0.0), (1.7976931348623157e308, 0.0), (1e-300, 1e-317),
        (123456789.0, 0.0), (0.1, 5.551115123125783e-18),
    ]
    # the reference test suite's curated sample values (test/unit/test.cc:112-155)
    samples = dd_from_mp([mpf(1) / 3, sqrt(2), pi, -e, 1 + mpf(2) ** -53, 1 - mpf(2) ** -54,
                          1 + mpf(2) ** -80, mpf(2) ** 100, mpf(2) ** -100, pi * mpf(2) ** 50,
                          -e * mpf(2) ** -50, mpf("-0.1")])
    base = np.concatenate([dd_list(common), samples])
    d = {}
    # exp: clamp and overflow/underflow rims (exp_log.inc:237-245), subnormal outputs
    em = 709.782712893384
    exp_edges = [em, np.nextafter(em, 1e9), np.nextafter(em, -1e9), -750.0, np.nextafter(-750.0, 0),
                 np.nextafter(-750.0, -1e9), -745.1, -744.4, -708.4, -708.3, 708.0, 1e-20, -1e-20,
                 0.34657359, -0.34657359, 0.693147180559945, 50.5, -50.5, 1.0 / 512, 1.0 / 256]
    d["exp"] = np.concatenate([base, W.with_lo(np.array(exp_edges), np.random.default_rng(7))])
    # log: near-1 branch boundaries (15/16, 17/16), negatives, subnormals, huge
    lg = [15 / 16, np.nextafter(15 / 16, 0), np.nextafter(15 / 16, 2), 17 / 16,
          np.nextafter(17 / 16, 0), np.nextafter(17 / 16, 2), 1 + 1e-12, 1 - 1e-12, 1e-310, 4e-320,
          -2.0, 1e308, 0.75, 1.5, 1.96875, 1.03125, 1.0 + 2 ** -52]
    d["log"] = np.concatenate([base, W.with_lo(np.array(lg), np.random.default_rng(8))])
    # trig: pi/8 branch, multiples of pi/2, the 2^55 cap, large arguments
    tr = [0.392699081698724, np.nextafter(0.392699081698724, 1), 0.7853981633974483,
          1.5707963267948966, 3.141592653589793, 4.71238898038469, -1.5707963267948966,
          2.0 ** 55, np.nextafter(2.0 ** 55, 0), -(2.0 ** 54), 1e15, 1e6, 47.15, 1e-8, -1e-8,
          355.0, 103993.0, 1e-300]
    tr_dd = dd_from_mp([k * pi / 2 for k in (1, 2, 3, 4, 15, 100, 10001, 636619)])
    d["sin"] = d["cos"] = np.concatenate([base, W.with_lo(np.array(tr), np.random.default_rng(9)), tr_dd])
    d["sqrt"] = np.concatenate([base, W.with_lo(np.array([4.0, 2.0, 1e-310, 1e308, 0.25, 1e-320, -4.0]),
                                                 np.random.default_rng(10))])
    # exp2: clamp rims exp2_max = 1024 - 2^-42 and exp2_min = -1080 (exp_log.inc:119-128),
    # subnormal outputs below 2^-1022, integer and half-integer arguments
    e2max, e2min = 1024.0 - 2.0 ** -42, -1080.0
    e2 = [e2max, np.nextafter(e2max, 2e3), np.nextafter(e2max, 0), 1024.0, 1023.5, e2min,
          np.nextafter(e2min, 0), np.nextafter(e2min, -2e3), -1074.0, -1074.5, -1075.0, -1022.0,
          -1022.5, -1023.0, 0.5, -0.5, 1.5, 10.0, -10.0, 1e-20, -1e-20, 0.25, 100.49999999999999]
    d["exp2"] = np.concatenate([base, W.with_lo(np.array(e2), np.random.default_rng(11))])
    d["log2"] = d["log10"] = d["log"]
    return d


def cexp_edges() -> np.ndarray:
    """complex64x2 arguments over the special-value grid of C99 Annex G.6.3.1
    (src/complex64x2/std.inc:20-74) plus ordinary and extreme finite ones."""
    inf, nan = float("inf"), float("nan")
    re_parts = [0.0, -0.0, 1.0, -1.0, 700.0, -750.0, 709.9, 1e-300, inf, -inf, nan]
    im_parts = [0.0, -0.0, 1.0, 1.5707963267948966, 3.141592653589793, 1e6, -2.5, 2.0 ** 56, inf, -inf, nan]
    rows = []
    for a in re_parts:
        for b in im_parts:
            rows.append([a, 0.0, b, 0.0])
    return np.array(rows, dtype=np.float64).reshape(-1)


def fuzz_mix(n: int, seed: int) -> np.ndarray:
    """The reference fuzz generator's mix (test/unit/test_common.hh:82-160), restated:
    10% non-finite, 10% close pairs, 10% cancelling pairs, 10% near-huge,
    10% near-tiny, 50% wide 10^[-30, 30]."""
    rng = np.random.default_rng(seed)
    r1, r2, r3 = rng.random(n), rng.random(n), rng.random(n)
    mode = (r1 * 10).astype(int)
    hi = (r2 - 0.5) * 10.0 ** ((r3 * 60).astype(int) - 30)
    nonfin = np.array([np.inf, -np.inf, np.nan, 0.0, -0.0])
    hi = np.where(mode == 0, nonfin[(r2 * 5).astype(int) % 5], hi)
    hi = np.where(mode == 3, (r2 - 0.5) * 2 * 10.0 ** ((r3 * 10).astype(int) + 20), hi)
    hi = np.where(mode == 4, (r2 - 0.5) * 2 * 10.0 ** (-((r3 * 10).astype(int) + 20)), hi)
    out = W.with_lo(np.where(np.isfinite(hi), hi, 0.0), rng)
    out[0::2] = np.where(np.isfinite(hi), out[0::2], hi)
    out[1::2] = np.where(np.isfinite(hi), out[1::2], 0.0)
    return out


GEMM_SHAPES = [
    # test/unit/fuzz.cc:1959-2016 and test/unit/precision.f90:928-946 shapes, ri = 8
    (1, 1, 1, 8), (7, 1, 9, 8), (3, 9, 1, 8), (2, 20, 5, 8), (16, 16, 16, 8), (4, 32, 6, 8),
    (3, 5, 2, 8), (3, 1, 2, 8), (1, 5, 1, 8), (1, 5, 7, 8), (7, 5, 1, 8), (5, 1, 1, 8),
    # renorm cadence edges: k < ri, k == ri, k == ri + 1, ri = 0, ri = 1, odd ri
    (9, 7, 5, 8), (9, 8, 5, 8), (9, 9, 5, 8), (33, 40, 17, 0), (12, 13, 11, 1), (20, 50, 21, 3),
    # tile edges of the device kernel (64 x 64 CTA tiles, k-tiles of 8)
    (65, 33, 70, 8), (128, 64, 64, 8), (63, 17, 129, 8),
]


def main() -> int:
    if not O.ref_available():
        print("oracle/_ref/libmfref.so not built; run `make -C oracle` where the reference exists")
        return 1
    g: dict[str, np.ndarray] = {}
    edges = edge_inputs()
    for op, gen in W.ELEMENTWISE_INPUTS.items():
        x = np.concatenate([edges[op], gen(2000, seed=100 + O.OPS[op]), fuzz_mix(600, 200 + O.OPS[op])])
        g[f"unary_{op}_x"] = x
        g[f"unary_{op}_y"] = O.ref_unary(op, x)
    # exp2 / log2 / log10 over their edges, the config-like distributions and the fuzz mix
    for op, gen in W.EXTRA_ELEMENTWISE_INPUTS.items():
        x = np.concatenate([edges[op], gen(2000, seed=100 + O.OPS[op]), fuzz_mix(600, 200 + O.OPS[op])])
        g[f"unary_{op}_x"] = x
        g[f"unary_{op}_y"] = O.ref_unary(op, x)
    # fused sincos and cexpi over the trig edges and distribution; cexp over the Annex G grid
    x = np.concatenate([edges["sin"], W.ELEMENTWISE_INPUTS["sin"](2000, seed=150), fuzz_mix(600, 250)])
    g["pair_sincos_x"] = x
    g["pair_sincos_s"], g["pair_sincos_c"] = O.ref_pair("sincos", x)
    g["pair_cexpi_x"] = x
    g["pair_cexpi_z"] = O.ref_pair("cexpi", x)
    rng = np.random.default_rng(151)
    z = np.concatenate([cexp_edges(),
                        W.complex_from_parts(W.with_lo(rng.uniform(-700.0, 700.0, 2000), rng),
                                             W.ELEMENTWISE_INPUTS["sin"](2000, seed=152)),
                        W.complex_from_parts(fuzz_mix(600, 253), fuzz_mix(600, 254))])
    g["pair_cexp_x"] = z
    g["pair_cexp_w"] = O.ref_pair("cexp", z)
    a = fuzz_mix(3000, 300)
    b = fuzz_mix(3000, 301)
    g["binary_a"], g["binary_b"] = a, b
    for op in range(4):
        g[f"binary_{op}_y"] = O.ref_binary(op, a, b)
    shapes = np.array(GEMM_SHAPES, dtype=np.int64)
    g["gemm_shapes"] = shapes
    for idx, (m, k, n, ri) in enumerate(GEMM_SHAPES):
        A = W.dd_uniform(m * k, seed=1000 + idx)
        B = W.dd_uniform(k * n, seed=2000 + idx)
        g[f"gemm{idx}_a"], g[f"gemm{idx}_b"] = A, B
        g[f"gemm{idx}_c"] = O.ref_matmul_mm(A, B, m, k, n, ri)
        g[f"gemm{idx}_mv"] = O.ref_matmul_mv(A, B[: 2 * k], m, k, ri)
        g[f"gemm{idx}_vm"] = O.ref_matmul_vm(A[: 2 * k], B, k, n, ri)
        if m * k * n <= 70000:
            CA = W.complex_from_parts(A, W.dd_uniform(m * k, seed=3000 + idx))
            CB = W.complex_from_parts(B, W.dd_uniform(k * n, seed=4000 + idx))
            g[f"cgemm{idx}_a"], g[f"cgemm{idx}_b"] = CA, CB
            g[f"cgemm{idx}_c"] = O.ref_cmatmul_mm(CA, CB, m, k, n, ri)
    for idx, n in enumerate([0, 1, 7, 1000, 5000]):
        x = W.dd_uniform(n, seed=5000 + idx)
        g[f"norm2_{idx}_x"] = x
        g[f"norm2_{idx}_y"] = O.ref_norm2(x)
    np.savez_compressed(OUT, **g)
    print(f"wrote {OUT} ({os.path.getsize(OUT)} bytes, {len(g)} arrays)")
    return 0


if __name__ == "__main__":
    sys.exit(main())
