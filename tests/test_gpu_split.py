"""GPU parity of the split-INT8 DD GEMM (tcgen05 INT8 tensor cores).

The integer stage is exact and the DD recombination has a fixed order, so the
device result is bit-identical to the CPU restatement of the same algorithm
(oracle.split_gemm); against the exact product it must stay within the stated
bound err_ij <= 8 k 2^-104 (|A||B|)_ij (and is far inside it)."""
import ctypes as C

import numpy as np
import pytest

from conftest import to_dev, to_host
from multifloats_b200 import _lib
from multifloats_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu
ULP = 2.0 ** -104


def dev_split(L, dev, A, B, m, k, n, slices=0, target=8.0):
    import torch

    a, b = to_dev(A, dev), to_dev(B, dev)
    c = torch.empty(2 * m * n, dtype=torch.float64, device=dev)
    info = (C.c_int * 3)()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = L.mfcuda_matmuldd_mm_split(a.data_ptr(), b.data_ptr(), c.data_ptr(), m, k, n, slices, target,
                                    None, 0, info, stream)
    assert rc == 0, _lib.lib().mfcuda_error_string(rc)
    return to_host(c), tuple(info)


def test_smallest_tile_bit_exact(cuda_lib, dev):
    m = k = n = 128
    A = W.dd_rowcol_scaled(m, k, 0, "row", seed=1)
    B = W.dd_rowcol_scaled(k, n, 0, "col", seed=2)
    got, info = dev_split(cuda_lib, dev, A, B, m, k, n)
    want, winfo = O.split_gemm(A, B, m, k, n)
    assert info == winfo
    assert O.same_bits(got, want).all(), np.count_nonzero(~O.same_bits(got, want))


@pytest.mark.parametrize("shape", [(256, 256, 256), (130, 300, 257), (1, 1, 1), (7, 129, 9),
                                   (300, 64, 520), (64, 1000, 16)])
@pytest.mark.parametrize("R", [0, 16, 64])
def test_bit_exact_vs_cpu_restatement(cuda_lib, dev, shape, R):
    m, k, n = shape
    A = W.dd_rowcol_scaled(m, k, R, "row", seed=m + R)
    B = W.dd_rowcol_scaled(k, n, R, "col", seed=n + R)
    got, info = dev_split(cuda_lib, dev, A, B, m, k, n)
    want, winfo = O.split_gemm(A, B, m, k, n)
    assert info == winfo
    assert O.same_bits(got, want).all()


@pytest.mark.parametrize("S", [2, 7, 12, 13, 14])
def test_fixed_slice_counts(cuda_lib, dev, S):
    m, k, n = 96, 200, 80
    A, B = W.dd_uniform(m * k, seed=S), W.dd_uniform(k * n, seed=S + 50)
    got, info = dev_split(cuda_lib, dev, A, B, m, k, n, slices=S)
    want, winfo = O.split_gemm(A, B, m, k, n, slices=S)
    assert info[0] == S and info == winfo
    assert O.same_bits(got, want).all()


def test_k_chunks(cuda_lib, dev):
    """k above one INT32-safe chunk (73*128) runs several K chunks."""
    m, k, n = 128, 20000, 64
    A = W.dd_rowcol_scaled(m, k, 4, "row", seed=3)
    B = W.dd_rowcol_scaled(k, n, 4, "col", seed=4)
    got, _ = dev_split(cuda_lib, dev, A, B, m, k, n)
    want, _ = O.split_gemm(A, B, m, k, n)
    assert O.same_bits(got, want).all()


@pytest.mark.parametrize("R", [0, 16, 64])
def test_error_bound_1024(cuda_lib, dev, R):
    m = k = n = 1024
    A = W.dd_rowcol_scaled(m, k, R, "row", seed=11)
    B = W.dd_rowcol_scaled(k, n, R, "col", seed=12)
    got, info = dev_split(cuda_lib, dev, A, B, m, k, n)
    rng = np.random.default_rng(R)
    ii, jj = rng.integers(0, m, 400), rng.integers(0, n, 400)
    err, ab = O.gemm_errors(A, B, got, m, k, n, ii, jj)
    ratio = np.abs(err) / (k * ULP * ab)
    assert ratio.max() <= 8.0, ratio.max()
    # it is in fact within a fraction of one DD ulp of |A||B|
    assert (np.abs(err) / (ULP * ab)).max() <= 1.0


def test_nonfinite_rows_give_nan(cuda_lib, dev):
    m, k, n = 64, 64, 64
    A, B = W.dd_uniform(m * k, seed=5), W.dd_uniform(k * n, seed=6)
    A[2 * (10 * m + 3)] = np.inf  # row 3 of A
    B[2 * (7 * k + 20)] = np.nan  # column 7 of B
    got, _ = dev_split(cuda_lib, dev, A, B, m, k, n)
    want, _ = O.split_gemm(A, B, m, k, n)
    assert O.same_bits(got, want).all()
    g = got.reshape(n, m, 2)
    assert np.isnan(g[:, 3, 0]).all() and np.isnan(g[7, :, 0]).all()
    assert np.isfinite(g[0, 0, 0])


def test_zero_matrix_and_k_zero(cuda_lib, dev):
    m, k, n = 40, 50, 30
    got, _ = dev_split(cuda_lib, dev, np.zeros(2 * m * k), W.dd_uniform(k * n, seed=1), m, k, n)
    assert np.all(got == 0.0)
    import torch

    c = torch.full((2 * m * n,), 7.0, dtype=torch.float64, device=dev)
    rc = cuda_lib.mfcuda_matmuldd_mm_split(None, None, c.data_ptr(), m, 0, n, 0, 8.0, None, 0, None, None)
    assert rc == 0 and np.all(to_host(c) == 0.0)


def test_host_dropin_split(cuda_lib):
    m, k, n = 200, 150, 120
    A = W.dd_rowcol_scaled(m, k, 16, "row", seed=7)
    B = W.dd_rowcol_scaled(k, n, 16, "col", seed=8)
    c = np.empty(2 * m * n)
    bound = C.c_double(-1.0)
    cuda_lib.matmuldd_mm_split(A.ctypes.data, B.ctypes.data, c.ctypes.data, m, k, n, 0, C.byref(bound))
    assert cuda_lib.mfcuda_last_error() == 0
    want, info = O.split_gemm(A, B, m, k, n)
    assert O.same_bits(c, want).all()
    assert 0.0 < bound.value <= 8.0  # S = 14, rho = 1: 15/16


def test_invalid_split_arguments(cuda_lib):
    assert cuda_lib.mfcuda_matmuldd_mm_split(None, None, None, -1, 2, 2, 0, 8.0, None, 0, None, None) == 1
    assert cuda_lib.mfcuda_matmuldd_mm_split(None, None, None, 2, 2, 2, 15, 8.0, None, 0, None, None) == 1
    assert cuda_lib.mfcuda_matmuldd_mm_split(None, None, None, 2, 2, 2, 0, 0.0, None, 0, None, None) == 1


# ---- complex64x2 split form (four real products, Fortran composition) ----
def _cplx(m, k, R, per, seed):
    return W.complex_from_parts(W.dd_rowcol_scaled(m, k, R, per, seed),
                                W.dd_rowcol_scaled(m, k, R, per, seed + 1000))


def dev_csplit(L, dev, A, B, m, k, n, slices=0):
    import torch

    a, b = to_dev(A, dev), to_dev(B, dev)
    c = torch.empty(4 * m * n, dtype=torch.float64, device=dev)
    info = (C.c_int * 3)()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = L.mfcuda_cmatmuldd_mm_split(a.data_ptr(), b.data_ptr(), c.data_ptr(), m, k, n, slices, 8.0,
                                     None, 0, info, stream)
    assert rc == 0, rc
    return to_host(c), tuple(info)


def _embed(A, B, m, k, n):
    """Exact real embeddings: Re(AB) = [Ar | -Ai][Br; Bi], Im(AB) = [Ar | Ai][Bi; Br]
    (column-major, DD interleaved)."""
    a = A.reshape(k, m, 4)
    b = B.reshape(n, k, 4)
    ar, ai = a[..., 0:2], a[..., 2:4]
    br, bi = b[..., 0:2], b[..., 2:4]
    a_re = np.concatenate([ar, -ai], axis=0).reshape(-1)
    a_im = np.concatenate([ar, ai], axis=0).reshape(-1)
    b_re = np.concatenate([br, bi], axis=1).reshape(-1)
    b_im = np.concatenate([bi, br], axis=1).reshape(-1)
    return (a_re, b_re), (a_im, b_im)


@pytest.mark.parametrize("shape", [(64, 100, 48), (130, 200, 257), (1, 3, 1)])
def test_complex_split_bit_exact(cuda_lib, dev, shape):
    m, k, n = shape
    A, B = _cplx(m, k, 16, "row", 1), _cplx(k, n, 16, "col", 2)
    got, info = dev_csplit(cuda_lib, dev, A, B, m, k, n)
    want, winfo = O.split_cgemm(A, B, m, k, n)
    assert info == winfo
    assert O.same_bits(got, want).all()


def test_complex_split_error_bound(cuda_lib, dev):
    m, k, n = 256, 512, 192
    A, B = _cplx(m, k, 16, "row", 3), _cplx(k, n, 16, "col", 4)
    got, _ = dev_csplit(cuda_lib, dev, A, B, m, k, n)
    g = got.reshape(n, m, 4)
    rng = np.random.default_rng(0)
    ii, jj = rng.integers(0, m, 200), rng.integers(0, n, 200)
    for part, (ae, be) in enumerate(_embed(A, B, m, k, n)):
        cpart = np.ascontiguousarray(g[..., 2 * part: 2 * part + 2]).reshape(-1)
        err, ab = O.gemm_errors(ae, be, cpart, m, 2 * k, n, ii, jj)
        assert (np.abs(err) / (k * ULP * ab)).max() <= 8.0
        assert (np.abs(err) / (ULP * ab)).max() <= 1.0


def test_complex_split_host_dropin(cuda_lib):
    m, k, n = 70, 90, 50
    A, B = _cplx(m, k, 4, "row", 5), _cplx(k, n, 4, "col", 6)
    c = np.empty(4 * m * n)
    bound = C.c_double(-1.0)
    cuda_lib.cmatmuldd_mm_split(A.ctypes.data, B.ctypes.data, c.ctypes.data, m, k, n, 0, C.byref(bound))
    assert cuda_lib.mfcuda_last_error() == 0
    want, _ = O.split_cgemm(A, B, m, k, n)
    assert O.same_bits(c, want).all()
    assert 0.0 < bound.value <= 8.0
