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
