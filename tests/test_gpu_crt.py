"""GPU parity of the CRT (modular) split-INT8 DD GEMM.

The device recovers the exact integer product of the rounded operands from
its residues modulo N moduli (one INT8 tensor-core product per modulus) and
rounds it to DD; the oracle computes the same exact integer directly with a
256-bit accumulator and applies the same rounding, so the results must match
bit for bit -- which also checks the modular reconstruction.  Against the
exact product the error stays within the stated bound err_ij <= 8 k 2^-104
(|A||B|)_ij."""
import ctypes as C

import numpy as np
import pytest

from conftest import to_dev, to_host
from multifloats_b200 import _lib
from multifloats_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu
ULP = 2.0 ** -104


def dev_crt(L, dev, A, B, m, k, n, bits=0, target=8.0, a=None, b=None):
    import torch

    a = to_dev(A, dev) if a is None else a
    b = to_dev(B, dev) if b is None else b
    c = torch.empty(2 * m * n, dtype=torch.float64, device=dev)
    info = (C.c_int * 4)()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = L.mfcuda_matmuldd_mm_crt(a.data_ptr(), b.data_ptr(), c.data_ptr(), m, k, n, bits, target,
                                  None, 0, info, stream)
    assert rc == 0, _lib.lib().mfcuda_error_string(rc)
    return to_host(c), list(info)


@pytest.mark.parametrize("shape", [(128, 128, 128), (256, 256, 256), (130, 300, 257), (1, 1, 1), (7, 129, 9),
                                   (300, 64, 520), (64, 1000, 16), (40, 9500, 24)])
@pytest.mark.parametrize("R", [0, 16, 64])
def test_bit_exact_vs_restatement(cuda_lib, dev, shape, R):
    m, k, n = shape
    A = W.dd_rowcol_scaled(m, k, R, "row", seed=m + R + 3)
    B = W.dd_rowcol_scaled(k, n, R, "col", seed=n + R + 4)
    got, info = dev_crt(cuda_lib, dev, A, B, m, k, n)
    want, winfo = O.crt_gemm(A, B, m, k, n)
    assert info == winfo
    ok = O.same_bits(got, want)
    assert ok.all(), (np.count_nonzero(~ok), np.flatnonzero(~ok)[:5])


@pytest.mark.parametrize("bits", [8, 40, 77, 110])
def test_fixed_bits(cuda_lib, dev, bits):
    m, k, n = 96, 200, 300
    A, B = W.dd_uniform(m * k, seed=bits), W.dd_uniform(k * n, seed=bits + 50)
    got, info = dev_crt(cuda_lib, dev, A, B, m, k, n, bits=bits)
    want, winfo = O.crt_gemm(A, B, m, k, n, bits=bits)
    assert info == winfo and info[3] == bits
    assert O.same_bits(got, want).all()


def test_nonfinite_zero_rows_and_wide_spread(cuda_lib, dev):
    """Inf/NaN in a row of A or column of B -> NaN outputs there; zero rows
    and columns -> exact zeros; entries spanning 2^+-300 within a row (the
    plan raises W, and at W = 110 reports a bound above the target)."""
    m, k, n = 150, 90, 270
    A = W.dd_uniform(m * k, seed=5).reshape(k, m, 2)
    B = W.dd_uniform(k * n, seed=6).reshape(n, k, 2)
    A[3, 7] = (np.inf, 0.0)
    A[:, 11] = 0.0
    A[10, 20] = (np.nan, 0.0)
    B[5, 40] = (-np.inf, 0.0)
    B[33] = 0.0
    A[:, 50] *= np.exp2(np.linspace(-300, 300, k))[:, None]
    A, B = A.reshape(-1), B.reshape(-1)
    got, info = dev_crt(cuda_lib, dev, A, B, m, k, n)
    want, winfo = O.crt_gemm(A, B, m, k, n)
    assert info == winfo
    assert O.same_bits(got, want).all()
    g = got.reshape(n, m, 2)
    assert np.isnan(g[:, 7, 0]).all() and np.isnan(g[:, 20, 0]).all() and np.isnan(g[5, :, 0]).all()
    assert (g[33, [0, 1, 2], :] == 0).all() and (g[[0, 1], 11, :] == 0).all()


def test_k_zero_and_empty(cuda_lib, dev):
    import torch

    m, n = 5, 7
    c = torch.full((2 * m * n,), 3.0, dtype=torch.float64, device=dev)
    assert cuda_lib.mfcuda_matmuldd_mm_crt(None, None, c.data_ptr(), m, 0, n, 0, 8.0, None, 0, None, None) == 0
    assert (to_host(c) == 0).all()
    assert cuda_lib.mfcuda_matmuldd_mm_crt(None, None, None, 0, 5, 5, 0, 8.0, None, 0, None, None) == 0
    # invalid: negative size, bits out of range, non-positive target
    assert cuda_lib.mfcuda_matmuldd_mm_crt(None, None, None, -1, 2, 2, 0, 8.0, None, 0, None, None) == 1
    assert cuda_lib.mfcuda_matmuldd_mm_crt(None, None, None, 2, 2, 2, 111, 8.0, None, 0, None, None) == 1
    assert cuda_lib.mfcuda_matmuldd_mm_crt(None, None, None, 2, 2, 2, 0, 0.0, None, 0, None, None) == 1


def test_unaligned_is_rejected_and_workspace(cuda_lib, dev):
    import torch

    m = k = n = 16
    a = torch.zeros(2 * m * k + 1, dtype=torch.float64, device=dev)[1:]
    b = torch.zeros(2 * k * n, dtype=torch.float64, device=dev)
    c = torch.zeros(2 * m * n, dtype=torch.float64, device=dev)
    assert cuda_lib.mfcuda_matmuldd_mm_crt(a.data_ptr(), b.data_ptr(), c.data_ptr(), m, k, n, 0, 8.0,
                                           None, 0, None, None) == 7  # MFCUDA_ERR_UNSUPPORTED
    A, B = W.dd_uniform(m * k, seed=1), W.dd_uniform(k * n, seed=2)
    ws_bytes = cuda_lib.mfcuda_crt_workspace_size(m, k, n, 0)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
    da, db = to_dev(A, dev), to_dev(B, dev)
    rc = cuda_lib.mfcuda_matmuldd_mm_crt(da.data_ptr(), db.data_ptr(), c.data_ptr(), m, k, n, 0, 8.0,
                                         ws.data_ptr(), ws_bytes - 1, None, None)
    assert rc == 6  # MFCUDA_ERR_WORKSPACE
    rc = cuda_lib.mfcuda_matmuldd_mm_crt(da.data_ptr(), db.data_ptr(), c.data_ptr(), m, k, n, 0, 8.0,
                                         ws.data_ptr(), ws_bytes, None, None)
    assert rc == 0
    want, _ = O.crt_gemm(A, B, m, k, n)
    assert O.same_bits(to_host(c), want).all()


def test_host_dropin(cuda_lib):
    m, k, n = 70, 130, 90
    A, B = W.dd_rowcol_scaled(m, k, 16, "row", 8), W.dd_rowcol_scaled(k, n, 16, "col", 9)
    c = np.empty(2 * m * n)
    bound = C.c_double()
    cuda_lib.matmuldd_mm_crt(A.ctypes.data, B.ctypes.data, c.ctypes.data, m, k, n, 0, C.byref(bound))
    assert cuda_lib.mfcuda_last_error() == 0
    want, info = O.crt_gemm(A, B, m, k, n)
    assert O.same_bits(c, want).all()
    assert bound.value == pytest.approx(O.crt_bound(info[3], info[1], info[2], k)) and bound.value <= 8.0


def test_host_dropin_column_panels(cuda_lib, dev):
    """The host-pointer call computes the output in column panels and copies
    each back while the next is computed: the same bits as the device call,
    with a ragged last panel (2100 columns: five 512-column tiles, one panel
    each, the last one 52 columns wide)."""
    m, k, n = 300, 700, 2100
    A, B = W.dd_rowcol_scaled(m, k, 16, "row", 18), W.dd_rowcol_scaled(k, n, 16, "col", 19)
    got, info = dev_crt(cuda_lib, dev, A, B, m, k, n)
    for _ in range(2):  # twice: the second call reuses the staging streams and events
        c = np.full(2 * m * n, np.nan)
        bound = C.c_double()
        cuda_lib.matmuldd_mm_crt(A.ctypes.data, B.ctypes.data, c.ctypes.data, m, k, n, 0, C.byref(bound))
        assert cuda_lib.mfcuda_last_error() == 0
        assert O.same_bits(c, got).all()
    want, _ = O.crt_gemm(A, B, m, k, n, rows=(150, 152))
    sub = np.ascontiguousarray(c.reshape(n, m, 2)[:, 150:152, :]).reshape(-1)
    assert O.same_bits(sub, want).all()


@pytest.mark.parametrize("R", [0, 16, 64])
def test_4096_error_bound_and_sampled_rows(cuda_lib, dev, R):
    """The benchmark shape: every sampled output within the a-priori bound of
    the exact product, and four full rows bit-identical to the restatement."""
    m = k = n = 4096
    A = W.dd_rowcol_scaled(m, k, R, "row", seed=101)
    B = W.dd_rowcol_scaled(k, n, R, "col", seed=102)
    got, info = dev_crt(cuda_lib, dev, A, B, m, k, n)
    assert (info[0], info[3]) == (26, 92)  # one binade per row / column: rho = 1
    bound = O.crt_bound(info[3], info[1], info[2], k)
    assert bound <= 8.0
    rng = np.random.default_rng(R)
    ii, jj = rng.integers(0, m, 256), rng.integers(0, n, 256)
    err, absv = O.gemm_errors(A, B, got, m, k, n, ii, jj)
    assert (np.abs(err) <= bound * k * ULP * absv).all()
    rows = (1000, 1004)
    want, _ = O.crt_gemm(A, B, m, k, n, rows=rows)
    sub = np.ascontiguousarray(got.reshape(n, m, 2)[:, rows[0]:rows[1], :]).reshape(-1)
    assert O.same_bits(sub, want).all()


@pytest.mark.parametrize("shape", [(96, 130, 64), (300, 200, 520), (1, 3, 2)])
def test_complex_bit_exact_and_host(cuda_lib, dev, shape):
    """Complex CRT form: four real products with one plan (from all four
    parts), combined re = ArBr - AiBi, im = ArBi + AiBr."""
    import torch

    m, k, n = shape
    A = W.complex_from_parts(W.dd_rowcol_scaled(m, k, 16, "row", 31), W.dd_rowcol_scaled(m, k, 16, "row", 32))
    B = W.complex_from_parts(W.dd_rowcol_scaled(k, n, 16, "col", 33), W.dd_rowcol_scaled(k, n, 16, "col", 34))
    a, b = to_dev(A, dev), to_dev(B, dev)
    c = torch.empty(4 * m * n, dtype=torch.float64, device=dev)
    info = (C.c_int * 4)()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = cuda_lib.mfcuda_cmatmuldd_mm_crt(a.data_ptr(), b.data_ptr(), c.data_ptr(), m, k, n, 0, 8.0, None, 0,
                                          info, stream)
    assert rc == 0
    want, winfo = O.crt_cgemm(A, B, m, k, n)
    assert list(info) == winfo
    assert O.same_bits(to_host(c), want).all()
    h = np.empty(4 * m * n)
    bound = C.c_double()
    cuda_lib.cmatmuldd_mm_crt(A.ctypes.data, B.ctypes.data, h.ctypes.data, m, k, n, 0, C.byref(bound))
    assert cuda_lib.mfcuda_last_error() == 0 and O.same_bits(h, want).all()


def test_column_panels_agree_on_width(cuda_lib, dev):
    """dist.CudaBackend.gemm_crt on three column panels of B (one process
    standing in for three ranks): each panel with its own width W, then all
    with the largest one, as dist.matmul_columns does; the panels together
    equal the single call bit for bit."""
    import torch

    from multifloats_b200 import dist as D

    m, k, n = 140, 300, 390
    A = W.dd_rowcol_scaled(m, k, 0, "row", seed=61)
    parts = [W.dd_rowcol_scaled(k, 130, 0, "col", seed=62), W.dd_rowcol_scaled(k, 130, 0, "col", seed=63),
             W.dd_rowcol_scaled(k, 130, 6, "row", seed=64)]  # the last panel spans several binades per column
    B = np.concatenate(parts)
    be = D.CudaBackend()
    a = to_dev(A, dev)
    own = [be.gemm_crt(a, to_dev(p, dev), m, k, 130, 0, 8.0)[1] for p in parts]
    w_all = max(own)
    assert len(set(own)) > 1
    panels = [be.gemm_crt(a, to_dev(p, dev), m, k, 130, w_all, 8.0) for p in parts]
    assert all(w == w_all for _, w in panels)
    got = to_host(torch.cat([c for c, _ in panels]))
    want, info = dev_crt(cuda_lib, dev, A, B, m, k, n)
    assert info[3] == w_all
    assert O.same_bits(got, want).all()


def test_python_api_split_forms_and_batch(cuda_lib, dev):
    """multifloats_b200.api: the split and CRT wrappers on host arrays and CUDA
    tensors, and GemmBatch, give the C ABI's bits."""
    import torch

    from multifloats_b200 import api

    m, k, n = 130, 170, 90
    A, B = W.dd_rowcol_scaled(m, k, 16, "row", 81), W.dd_rowcol_scaled(k, n, 16, "col", 82)
    want, winfo = O.crt_gemm(A, B, m, k, n)
    c, info = api.matmuldd_mm_crt(to_dev(A, dev), to_dev(B, dev), m, k, n)
    assert O.same_bits(to_host(c), want).all()
    assert [info["moduli"], info["rho_a"], info["rho_b"], info["bits"]] == winfo
    h, hinfo = api.matmuldd_mm_crt(A, B, m, k, n)
    assert O.same_bits(h, want).all() and hinfo["bound"] == pytest.approx(O.crt_bound(winfo[3], winfo[1], winfo[2], k))
    swant, sinfo = O.split_gemm(A, B, m, k, n)
    s, si = api.matmuldd_mm_split(to_dev(A, dev), to_dev(B, dev), m, k, n)
    assert O.same_bits(to_host(s), swant).all() and si["slices"] == sinfo[0]
    with pytest.raises(ValueError):
        api.matmuldd_mm_crt(A, B, m, k, n, target=4.0)  # host calls have the fixed target 8
    with pytest.raises(ValueError):  # a host operand beside a device one is refused, not dereferenced
        api.matmuldd_mm_crt(to_dev(A, dev), torch.from_numpy(B), m, k, n)
    Z = (W.complex_from_parts(A, W.dd_rowcol_scaled(m, k, 16, "row", 83)),
         W.complex_from_parts(B, W.dd_rowcol_scaled(k, n, 16, "col", 84)))
    zc, _ = api.cmatmuldd_mm_crt(to_dev(Z[0], dev), to_dev(Z[1], dev), m, k, n)
    assert O.same_bits(to_host(zc), O.crt_cgemm(Z[0], Z[1], m, k, n)[0]).all()
    shapes = [(m, k, n), (40, 300, 70), (1, 5, 3)]
    probs = []
    for i, (mm, kk, nn) in enumerate(shapes):
        a = to_dev(W.dd_uniform(mm * kk, seed=90 + i), dev)
        b = to_dev(W.dd_uniform(kk * nn, seed=95 + i), dev)
        probs.append((a, b, torch.empty(2 * mm * nn, dtype=torch.float64, device=dev), mm, kk, nn))
    with api.GemmBatch(probs, form="crt") as bt:
        bt.run()
        assert bt.status() == 0
        for a, b, cc, mm, kk, nn in probs:
            assert O.same_bits(to_host(cc), O.crt_gemm(to_host(a), to_host(b), mm, kk, nn)[0]).all()


def test_widest_plan_two_k_steps_in_reconstruction(cuda_lib, dev):
    """W = 110 with k = 300000 needs 33 moduli: the reconstruction's MMA takes
    two K steps of 32 moduli, its E matrix 48 columns, and the residues of 33
    K chunks are summed per modulus first."""
    m, k, n = 5, 300000, 7
    A, B = W.dd_uniform(m * k, seed=201), W.dd_uniform(k * n, seed=202)
    got, info = dev_crt(cuda_lib, dev, A, B, m, k, n, bits=110)
    want, winfo = O.crt_gemm(A, B, m, k, n, bits=110)
    assert info == winfo and info[0] == 33 and info[3] == 110
    assert O.same_bits(got, want).all()

