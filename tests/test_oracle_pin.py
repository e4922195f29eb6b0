"""Pin the oracle (the C restatement in oracle/mf_oracle.c) before trusting it:
against the golden vectors the reference library produced (always), and against
the reference library itself on fresh inputs (where it was built here)."""
import numpy as np
import pytest

from multifloats_b200 import workloads as W
from oracle import oracle as O

OPS = ["exp", "log", "sin", "cos", "sqrt", "exp2", "log2", "log10"]


@pytest.mark.parametrize("op", OPS)
def test_unary_vs_golden(golden, op):
    x, y = golden[f"unary_{op}_x"], golden[f"unary_{op}_y"]
    ok = O.same_bits(O.unary(op, x), y)
    assert ok.all(), f"{op}: {np.count_nonzero(~ok)} of {ok.size} differ"


def test_sincos_cexpi_cexp_vs_golden(golden):
    s, c = O.pair("sincos", golden["pair_sincos_x"])
    assert O.same_bits(s, golden["pair_sincos_s"]).all() and O.same_bits(c, golden["pair_sincos_c"]).all()
    assert O.same_bits(O.pair("cexpi", golden["pair_cexpi_x"]), golden["pair_cexpi_z"]).all()
    w = O.pair("cexp", golden["pair_cexp_x"])
    ok = O.same_bits(w, golden["pair_cexp_w"])
    assert ok.all(), f"cexp: {np.count_nonzero(~ok)} of {ok.size} differ"
    # the fused form equals the separate sine and cosine, bit for bit
    x = golden["pair_sincos_x"]
    assert O.same_bits(s, O.unary("sin", x)).all() and O.same_bits(c, O.unary("cos", x)).all()


@pytest.mark.parametrize("op", range(4))
def test_binary_ops_vs_golden(golden, op):
    y = O.binary(op, golden["binary_a"], golden["binary_b"])
    assert O.same_bits(y, golden[f"binary_{op}_y"]).all()


def test_gemm_vs_golden(golden):
    for idx, (m, k, n, ri) in enumerate(golden["gemm_shapes"]):
        m, k, n, ri = int(m), int(k), int(n), int(ri)
        a, b = golden[f"gemm{idx}_a"], golden[f"gemm{idx}_b"]
        assert O.same_bits(O.matmul_mm(a, b, m, k, n, ri), golden[f"gemm{idx}_c"]).all(), (m, k, n, ri)
        assert O.same_bits(O.matmul_mv(a, b[: 2 * k], m, k, ri), golden[f"gemm{idx}_mv"]).all()
        assert O.same_bits(O.matmul_vm(a[: 2 * k], b, k, n, ri), golden[f"gemm{idx}_vm"]).all()
        if f"cgemm{idx}_a" in golden.files:
            c = O.cmatmul_mm(golden[f"cgemm{idx}_a"], golden[f"cgemm{idx}_b"], m, k, n, ri)
            assert O.same_bits(c, golden[f"cgemm{idx}_c"]).all(), (m, k, n, ri)


def test_norm2_vs_golden(golden):
    for idx in range(5):
        x = golden[f"norm2_{idx}_x"]
        assert O.same_bits(O.reduce_serial("norm2", x), golden[f"norm2_{idx}_y"]).all()


needs_ref = pytest.mark.skipif(not O.ref_available(), reason="reference library not built here")


@needs_ref
@pytest.mark.parametrize("op", OPS)
def test_unary_vs_reference_fresh(op):
    x = {**W.ELEMENTWISE_INPUTS, **W.EXTRA_ELEMENTWISE_INPUTS}[op](50000, seed=777)
    assert O.same_bits(O.unary(op, x), O.ref_unary(op, x)).all()


@needs_ref
def test_gemm_vs_reference_fresh():
    rng = np.random.default_rng(5)
    for _ in range(12):
        m, k, n = (int(v) for v in rng.integers(1, 60, 3))
        ri = int(rng.choice([0, 1, 2, 5, 8, 16]))
        a, b = W.dd_uniform(m * k, seed=m + 100 * k), W.dd_uniform(k * n, seed=n + 7 * k)
        assert O.same_bits(O.matmul_mm(a, b, m, k, n, ri), O.ref_matmul_mm(a, b, m, k, n, ri)).all()


def test_wgemm_vs_golden(golden):
    from conftest import wgemm_golden

    n = 0
    for i, args, want in wgemm_golden(golden):
        info, got = O.wgemm(*args)
        assert info == 0 and O.same_bits(got, want).all(), (i, args[:5])
        n += 1
    assert n >= 90


def test_wtrsm_vs_golden(golden):
    from conftest import wtrsm_golden

    n = 0
    for i, args, want in wtrsm_golden(golden):
        info, got = O.wtrsm(*args)
        assert info == 0 and O.same_bits(got, want).all(), (i, args[:6])
        n += 1
    assert n >= 100


def test_blas_argument_checks():
    """The info codes of wgemm.f90:29-48 / wtrsm.f90:24-44, first failing check wins."""
    assert O.wgemm_info("N", "N", 2, 3, 4, 2, 4, 2) == 0
    assert O.wgemm_info("X", "Q", -1, 3, 4, 2, 4, 2) == 1
    assert O.wgemm_info("t", "Q", -1, 3, 4, 2, 4, 2) == 2
    assert O.wgemm_info("c", "n", -1, -3, 4, 2, 4, 2) == 3
    assert O.wgemm_info("N", "N", 2, -3, 4, 2, 4, 2) == 4
    assert O.wgemm_info("N", "N", 2, 3, -4, 2, 4, 2) == 5
    assert O.wgemm_info("N", "N", 2, 3, 4, 1, 4, 2) == 8
    assert O.wgemm_info("T", "N", 2, 3, 4, 3, 4, 2) == 8  # lda >= k when A is transposed
    assert O.wgemm_info("N", "N", 2, 3, 4, 2, 3, 2) == 10
    assert O.wgemm_info("N", "T", 2, 3, 4, 2, 2, 2) == 10  # ldb >= n when B is transposed
    assert O.wgemm_info("N", "N", 2, 3, 4, 2, 4, 1) == 13
    assert O.wgemm_info("N", "N", 0, 0, 0, 1, 1, 1) == 0  # max(1, .) floors
    assert O.wgemm_info("N", "N", 0, 0, 0, 0, 1, 1) == 8
    assert O.wtrsm_info("L", "U", "N", "N", 3, 2, 3, 3) == 0
    assert O.wtrsm_info("X", "U", "N", "N", 3, 2, 3, 3) == 1
    assert O.wtrsm_info("r", "X", "N", "N", 3, 2, 3, 3) == 2
    assert O.wtrsm_info("L", "l", "X", "N", 3, 2, 3, 3) == 3
    assert O.wtrsm_info("L", "U", "c", "X", 3, 2, 3, 3) == 4
    assert O.wtrsm_info("L", "U", "N", "u", -3, 2, 3, 3) == 5
    assert O.wtrsm_info("L", "U", "N", "N", 3, -2, 3, 3) == 6
    assert O.wtrsm_info("L", "U", "N", "N", 3, 2, 2, 3) == 9
    assert O.wtrsm_info("R", "U", "N", "N", 3, 2, 2, 3) == 0  # right side: lda >= n
    assert O.wtrsm_info("L", "U", "N", "N", 3, 2, 3, 2) == 11
    # an invalid call writes nothing
    c = np.full(8, 7.0)
    info, out = O.wgemm("N", "N", 2, 2, 2, [1.0, 0.0], np.ones(8), 1, np.ones(8), 2, [0.0, 0.0], c, 2)
    assert info == 8 and (out == 7.0).all()


@needs_ref
def test_blas_vs_reference_fresh():
    import sys, os

    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    from make_golden import wgemm_operands, wtrsm_operands

    rng = np.random.default_rng(77)
    for t in range(40):
        case = (str(rng.choice(list("NTC"))), str(rng.choice(list("NTC"))), *(int(v) for v in rng.integers(0, 30, 3)),
                *(int(v) for v in rng.integers(0, 3, 3)), str(rng.choice(["rand", "one", "zero", "two"])),
                str(rng.choice(["rand", "one", "zero", "negzero"])), int(rng.integers(0, 2)))
        args = wgemm_operands(case, 8000 + t)
        info, got = O.wgemm(*args)
        assert info == 0 and O.same_bits(got, O.ref_wgemm(*args)).all(), case
    for t in range(48):
        case = (str(rng.choice(list("LR"))), str(rng.choice(list("UL"))), str(rng.choice(list("NTC"))),
                str(rng.choice(list("NU"))), *(int(v) for v in rng.integers(0, 40, 2)),
                str(rng.choice(["rand", "one", "two"])), float(rng.choice([0.0, 0.3])), int(rng.integers(0, 2)))
        args = wtrsm_operands(case, 9000 + t)
        info, got = O.wtrsm(*args)
        assert info == 0 and O.same_bits(got, O.ref_wtrsm(*args)).all(), case
