"""The CRT form's restatement (the oracle the GPU results are compared with
bit for bit) checked on the CPU against exact products: every output lies
within the a-priori bound the plan reports, in units of k 2^-104 (|A||B|)_ij,
for uniform data, row / column exponent spreads, fixed operand widths, the
complex composition, zero rows and non-finite entries."""
import numpy as np
import pytest

from multifloats_b200 import workloads as W
from oracle import oracle as O

ULP = 2.0 ** -104


def _check(A, B, m, k, n, c, info, seed):
    bound = O.crt_bound(info[3], info[1], info[2], k)
    rng = np.random.default_rng(seed)
    ii, jj = rng.integers(0, m, 64), rng.integers(0, n, 64)
    err, absab = O.gemm_errors(A, B, c, m, k, n, ii, jj)
    assert (np.abs(err) <= bound * k * ULP * absab).all(), (info, np.max(np.abs(err) / (k * ULP * absab)))
    return bound


@pytest.mark.parametrize("R", [0, 16, 64])
def test_crt_restatement_within_bound(R):
    m, k, n = 40, 300, 30
    A = W.dd_rowcol_scaled(m, k, R, "row", seed=500 + R)
    B = W.dd_rowcol_scaled(k, n, R, "col", seed=600 + R)
    c, info = O.crt_gemm(A, B, m, k, n)
    assert _check(A, B, m, k, n, c, info, R) <= 8.0


@pytest.mark.parametrize("bits", [24, 60, 110])
def test_crt_restatement_fixed_width(bits):
    m, k, n = 17, 200, 23
    A, B = W.dd_uniform(m * k, seed=bits), W.dd_uniform(k * n, seed=bits + 1)
    c, info = O.crt_gemm(A, B, m, k, n, bits=bits)
    assert info[3] == bits
    _check(A, B, m, k, n, c, info, bits)
    # a wider operand never gives a larger error bound
    if bits < 110:
        assert O.crt_bound(bits + 1, info[1], info[2], k) <= O.crt_bound(bits, info[1], info[2], k)


def test_crt_restatement_zero_and_nonfinite():
    m, k, n = 12, 50, 9
    A = W.dd_uniform(m * k, seed=7).reshape(k, m, 2)
    B = W.dd_uniform(k * n, seed=8).reshape(n, k, 2)
    A[:, 3] = 0.0          # zero row of A
    A[10, 5] = (np.nan, 0.0)
    B[4, 7] = (np.inf, 0.0)
    A, B = A.reshape(-1), B.reshape(-1)
    c, info = O.crt_gemm(A, B, m, k, n)
    C = c.reshape(n, m, 2)
    assert np.isnan(C[:, 5, 0]).all() and np.isnan(C[4, :, 0]).all()
    assert (C[np.arange(n) != 4, 3] == 0.0).all()


def test_crt_restatement_complex():
    m, k, n = 11, 120, 13
    A = W.complex_from_parts(W.dd_rowcol_scaled(m, k, 16, "row", 41), W.dd_rowcol_scaled(m, k, 16, "row", 42))
    B = W.complex_from_parts(W.dd_rowcol_scaled(k, n, 16, "col", 43), W.dd_rowcol_scaled(k, n, 16, "col", 44))
    c, info = O.crt_cgemm(A, B, m, k, n)
    # real part Ar Br - Ai Bi, checked term by term against the real restatement
    Ar, Ai = A.reshape(-1, 4)[:, :2].reshape(-1), A.reshape(-1, 4)[:, 2:].reshape(-1)
    Br, Bi = B.reshape(-1, 4)[:, :2].reshape(-1), B.reshape(-1, 4)[:, 2:].reshape(-1)
    for x, y in ((Ar, Br), (Ai, Bi), (Ar, Bi), (Ai, Br)):
        cc, ii = O.crt_gemm(x, y, m, k, n, bits=info[3])
        _check(x, y, m, k, n, cc, ii, 3)
    assert np.isfinite(c).all()
