"""Generate tests/golden/golden.npz from the reference library itself.

Run in a checkout where the reference sources were compiled into
oracle/_ref/libmfref.so (``make -C oracle``):

    python tests/golden/make_golden.py

Every output stored here was computed by the reference's own exported
functions (expdd, logdd, sindd, cosdd, sqrtdd, exp2dd, log2dd, log10dd,
sincosdd, cexpidd, cexpdd, adddd..divdd, matmuldd_mm/mv/vm)
or by compositions of them that mirror the Fortran layer (complex matmul from
four matmuldd_mm calls and the DD operators; norm2 from the DD operators and
sqrtdd; the BLAS-style shims wgemm / wtrsm from the DD operators in the
Fortran's loop order).  Inputs are seeded and regenerable.  The fixtures let the tests pin
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


# BLAS-style shim cases: every branch of wgemm.f90 / wtrsm.f90 (quick returns,
# alpha = 0, beta = 0 / 1 / other, k = 0, both transpositions, padded leading
# dimensions, zero and non-finite entries).
_DDK = {"rand": None, "one": (1.0, 0.0), "zero": (0.0, 0.0), "negzero": (-0.0, 0.0),
        "onelo": (1.0, 2.0 ** -60), "two": (2.0, 0.0), "nan": (float("nan"), 0.0)}


def _dd_scalar(kind: str, rng) -> np.ndarray:
    if _DDK[kind] is None:
        return W.with_lo(rng.uniform(-2.0, 2.0, 1), rng)
    return np.array(_DDK[kind], dtype=np.float64)


def _sprinkle(x: np.ndarray, rng, count: int) -> None:
    """Put inf / -inf / NaN into `count` random (non-padding) entries."""
    v = x.reshape(-1, 2)
    ok = np.flatnonzero(~np.isnan(v[:, 0]))
    if ok.size == 0 or count == 0:
        return
    for i, val in zip(rng.choice(ok, min(count, ok.size), replace=False), [np.inf, -np.inf, np.nan] * count):
        v[i] = (val, 0.0)


def wgemm_cases():
    rng = np.random.default_rng(900)
    cases = []
    shapes = [(5, 4, 3), (17, 9, 33), (33, 17, 8), (1, 1, 1), (0, 3, 2), (4, 0, 2), (6, 5, 0), (24, 21, 40)]
    scal = [("rand", "rand"), ("rand", "zero"), ("rand", "one"), ("zero", "one"), ("zero", "zero"),
            ("zero", "rand"), ("negzero", "two"), ("onelo", "onelo"), ("one", "negzero"), ("nan", "rand")]
    idx = 0
    for ta in "NTC":
        for tb in "NTc":
            for s_i, (m, n, k) in enumerate(shapes):
                al, be = scal[(idx * 3 + s_i) % len(scal)]
                if s_i == 0:
                    al, be = scal[idx % len(scal)]
                cases.append((ta, tb, m, n, k, int(rng.integers(0, 3)), int(rng.integers(0, 3)),
                              int(rng.integers(0, 3)), al, be, 2 if s_i == 1 else 0))
                idx += 1
    # every scalar pair on one shape of each transposition of A
    for ta in "NT":
        for al, be in scal:
            cases.append((ta, "N", 9, 7, 11, 1, 0, 2, al, be, 0))
    return cases


def wtrsm_cases():
    cases = []
    for side in "LR":
        for uplo in "UL":
            for ta in "NTC":
                for diag in "NU":
                    for (m, n, al, zeros, special) in [(23, 9, "rand", 0.2, 0), (7, 31, "one", 0.4, 0),
                                                       (26, 19, "two", 0.0, 2), (1, 3, "onelo", 0.0, 0)]:
                        cases.append((side, uplo, ta, diag, m, n, al, zeros, special))
    cases += [("L", "U", "N", "N", 0, 4, "rand", 0.0, 0), ("R", "L", "T", "U", 5, 0, "rand", 0.0, 0),
              ("L", "L", "N", "N", 6, 5, "zero", 0.0, 0), ("R", "U", "N", "N", 6, 5, "negzero", 0.0, 0),
              ("l", "u", "t", "n", 8, 3, "nan", 0.0, 0)]
    return cases


def wgemm_operands(case, seed):
    ta, tb, m, n, k, pa, pb, pc, al, be, special = case
    rng = np.random.default_rng(seed)
    nota, notb = ta.upper() == "N", tb.upper() == "N"
    ra, ca = (m, k) if nota else (k, m)
    rb, cb = (k, n) if notb else (n, k)
    lda, ldb, ldc = max(1, ra) + pa, max(1, rb) + pb, max(1, m) + pc
    a = W.dd_padded(ra, ca, lda, seed, zeros=0.1)
    b = W.dd_padded(rb, cb, ldb, seed + 1, zeros=0.1)
    c = W.dd_padded(m, n, ldc, seed + 2)
    if special:
        _sprinkle(a, rng, special)
        _sprinkle(b, rng, special)
    return (ta, tb, m, n, k, _dd_scalar(al, rng), a, lda, b, ldb, _dd_scalar(be, rng), c, ldc)


def wtrsm_operands(case, seed):
    side, uplo, ta, diag, m, n, al, zeros, special = case
    rng = np.random.default_rng(seed)
    na = m if side.upper() == "L" else n
    lda, ldb = max(1, na) + int(rng.integers(0, 3)), max(1, m) + int(rng.integers(0, 3))
    a = W.dd_triangular(na, lda, seed, zeros=zeros)
    b = W.dd_padded(m, n, ldb, seed + 1, zeros=zeros)
    if special:
        _sprinkle(b, rng, special)
        _sprinkle(a, rng, 1)
    return (side, uplo, ta, diag, m, n, _dd_scalar(al, rng), a, lda, b, ldb)


def _letters(*xs) -> np.ndarray:
    return np.array([ord(x) for x in xs], dtype=np.int64)


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
    for idx, case in enumerate(wgemm_cases()):
        ta, tb, m, n, k, al, a, lda, b, ldb, be, c, ldc = wgemm_operands(case, 6000 + 10 * idx)
        g[f"wgemm{idx}_p"] = np.concatenate([_letters(ta, tb), [m, n, k, lda, ldb, ldc]]).astype(np.int64)
        g[f"wgemm{idx}_s"] = np.concatenate([al, be])
        g[f"wgemm{idx}_a"], g[f"wgemm{idx}_b"], g[f"wgemm{idx}_c"] = a, b, c
        g[f"wgemm{idx}_out"] = O.ref_wgemm(ta, tb, m, n, k, al, a, lda, b, ldb, be, c, ldc)
    for idx, case in enumerate(wtrsm_cases()):
        side, uplo, ta, diag, m, n, al, a, lda, b, ldb = wtrsm_operands(case, 7000 + 10 * idx)
        g[f"wtrsm{idx}_p"] = np.concatenate([_letters(side, uplo, ta, diag), [m, n, lda, ldb]]).astype(np.int64)
        g[f"wtrsm{idx}_s"] = al
        g[f"wtrsm{idx}_a"], g[f"wtrsm{idx}_b"] = a, b
        g[f"wtrsm{idx}_out"] = O.ref_wtrsm(side, uplo, ta, diag, m, n, al, a, lda, b, ldb)
    np.savez_compressed(OUT, **g)
    print(f"wrote {OUT} ({os.path.getsize(OUT)} bytes, {len(g)} arrays)")
    return 0


if __name__ == "__main__":
    sys.exit(main())
