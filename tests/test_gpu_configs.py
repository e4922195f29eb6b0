"""GPU parity at the sizes of the benchmark configurations themselves, not only
at test-sized shapes:

  * plain compensated GEMM at 4096^3: whole rows and columns bit-identical to
    the reference MAC order (oracle restatement of src/float64x2/matmul.inc:6-39,
    pinned to the reference's own outputs), sampled outputs within k 2^-104 (|A||B|)_ij;
  * every elementwise map over 2^26 elements of its config distribution,
    every element bit-identical to the oracle (exp_log.inc, trig.inc, float64x2.h);
  * sum / dot_product / norm2 over 2^26 elements and the complex kinds over 2^24,
    bit-identical to the restated blocked order and within the bound of the exact value;
  * the split-INT8 (CRT) product at 4096^3 for R in {0, 16, 64}, at 8192^3 and
    complex at 4096^3: the error of EVERY output, measured on the device against
    the plain product, within the 8 k 2^-104 (|A||B|)_ij target;
  * the 2000-problem uneven batch (M, N, K log-uniform in [16, 1024]) in the
    plain and CRT forms: every problem checked on sampled columns / rows;
  * 10^4 ragged exp / log arrays with lengths log-uniform in [64, 2^20].

The oracle runs on every host core (its C calls release the GIL)."""
import ctypes as C

import numpy as np
import pytest

from conftest import to_dev, to_host
from multifloats_b200 import accuracy, api
from multifloats_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu
ULP = 2.0 ** -104


def _stream():
    import torch

    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def test_plain_gemm_4096_rows_and_columns_bit_exact(dev):
    m = k = n = 4096
    a, b = W.dd_uniform(m * k, seed=40), W.dd_uniform(k * n, seed=41)
    c = to_host(api.matmuldd_mm(to_dev(a, dev), to_dev(b, dev), m, k, n, 8)).reshape(n, m, 2)
    rows = [0, 1, 1000, 2047, 2048, 3001, 4094, 4095]
    cols = [0, 1, 777, 2047, 2048, 3333, 4094, 4095]
    want_r = O.matmul_mm_rows(a, b, m, k, n, 8, rows)
    assert O.same_bits(np.stack([c[:, i, :] for i in rows]), want_r).all()
    want_c = O.matmul_mm_columns(a, b, m, k, n, 8, cols)
    assert O.same_bits(c[cols], want_c).all()
    rng = np.random.default_rng(4096)
    ii, jj = rng.integers(0, m, 256), rng.integers(0, n, 256)
    err, ab = O.gemm_errors(a, b, c.reshape(-1), m, k, n, ii, jj)
    assert np.all(np.abs(err) <= k * ULP * ab)


@pytest.mark.parametrize("op", list(W.ELEMENTWISE_INPUTS))
def test_elementwise_2_26_every_element(dev, op):
    n = 1 << 26
    x = W.ELEMENTWISE_INPUTS[op](n, seed=26)
    got = to_host(api.unary(op, to_dev(x, dev)))
    same = O.same_bits(got, O.unary(op, x, threads=0))
    assert same.all(), (op, int((~same).sum()), np.flatnonzero(~same)[:8])


@pytest.mark.parametrize("kind,n", [("sum", 1 << 26), ("dot", 1 << 26), ("norm2", 1 << 26),
                                    ("csum", 1 << 24), ("cdot", 1 << 24), ("cnorm2", 1 << 24)])
def test_reductions_at_config_size(dev, kind, n):
    per = 2 if kind.startswith("c") else 1
    x = W.dd_uniform(per * n, seed=60)
    y = W.dd_uniform(per * n, seed=61) if "dot" in kind else None
    fn = {"sum": api.sum_dd, "dot": api.dot_product, "norm2": api.norm2, "csum": api.csum_dd,
          "cdot": api.cdot_product, "cnorm2": api.cnorm2}[kind]
    dx = to_dev(x, dev)
    got = to_host(fn(dx, to_dev(y, dev)) if y is not None else fn(dx))
    want = O.reduce_blocked(kind, x, y, 8)
    assert O.same_bits(got, want).all(), (kind, got, want)
    if kind in ("sum", "dot"):  # within 16 2^-104 sum |x| (resp. |a||b|) of the exact value
        err, mag = O.reduce_error(kind, x, y, got)
        assert abs(err) <= 16 * ULP * mag


def _crt(L, dA, dB, dC, m, k, n, cplx=False):
    sym = L.mfcuda_cmatmuldd_mm_crt if cplx else L.mfcuda_matmuldd_mm_crt
    info = (C.c_int * 4)()
    assert sym(dA.data_ptr(), dB.data_ptr(), dC.data_ptr(), m, k, n, 0, 8.0, None, 0, info, _stream()) == 0
    return list(info)


@pytest.mark.parametrize("n,R", [(4096, 0), (4096, 16), (4096, 64), (8192, 16)])
def test_crt_error_of_every_output(cuda_lib, dev, n, R):
    """Config 3: max over ALL outputs of |C_crt - C_plain| / (k 2^-104 (|A||B|)_ij)
    stays below 7, so every output is within the 8 k-ulp target of the exact
    product (the plain product is within 1 of it); 256 sampled outputs are
    also checked against the exact product directly."""
    import torch

    a = W.dd_rowcol_scaled(n, n, R, "row", 70 + R)
    b = W.dd_rowcol_scaled(n, n, R, "col", 80 + R)
    dA, dB = to_dev(a, dev), to_dev(b, dev)
    dC = torch.empty_like(dA)
    moduli, ra, rb, bits = _crt(cuda_lib, dA, dB, dC, n, n, n)
    bound = cuda_lib.mfcuda_crt_bound(bits, ra, rb, n)
    assert 0 < bound <= 8.0
    st = accuracy.full_error_real(dA, dB, dC, n, n, n)
    assert st["nonfinite_outputs"] == 0 and st["nonzero_where_absab_zero"] == 0
    assert st["max_err_vs_plain_k_ulp_absab"] < min(7.0, bound + 1.0), st
    rng = np.random.default_rng(n + R)
    ii, jj = rng.integers(0, n, 256), rng.integers(0, n, 256)
    err, ab = O.gemm_errors(a, b, to_host(dC), n, n, n, ii, jj)
    assert np.all(np.abs(err) <= bound * n * ULP * ab)


def test_complex_crt_error_of_every_output(cuda_lib, dev):
    """Config 5: complex 4096^3 in the CRT form (four real products), error of
    every output per part against the plain complex product."""
    import torch

    n = 4096
    a = W.complex_from_parts(W.dd_rowcol_scaled(n, n, 16, "row", 91), W.dd_rowcol_scaled(n, n, 16, "row", 92))
    b = W.complex_from_parts(W.dd_rowcol_scaled(n, n, 16, "col", 93), W.dd_rowcol_scaled(n, n, 16, "col", 94))
    dA, dB = to_dev(a, dev), to_dev(b, dev)
    dC = torch.empty_like(dA)
    _crt(cuda_lib, dA, dB, dC, n, n, n, cplx=True)
    st = accuracy.full_error_complex(dA, dB, dC, n, n, n)
    for part in ("re", "im"):
        assert st[part]["nonfinite_outputs"] == 0
    assert st["max_err_vs_plain_k_ulp_absab"] < 7.0, st


def _config4_shapes(count=2000, seed=2024):
    rng = np.random.default_rng(seed)
    return [tuple(int(v) for v in s) for s in np.exp(rng.uniform(np.log(16), np.log(1024), (count, 3)))]


def test_batch_2000_uneven_plain_and_crt(cuda_lib, dev):
    """Config 4: 2000 GEMMs with M, N, K log-uniform in [16, 1024], entries as
    config 1, one grouped launch per form.  Plain: two columns of every problem
    bit-identical to the reference MAC order.  CRT: one row of every problem
    bit-identical to the CRT restatement."""
    from test_gpu_batched import Batch

    shapes = _config4_shapes()
    bt = Batch(cuda_lib, dev, shapes, 7000, W.dd_uniform)
    rng = np.random.default_rng(5)
    picks = [(int(rng.integers(0, n)), int(rng.integers(0, n)), int(rng.integers(0, m))) for m, _, n in shapes]
    for form in (0, 2):
        p = bt.plan(form)
        try:
            bt.run(p)
            got = [to_host(bt.C[i]).reshape(shapes[i][2], shapes[i][0], 2) for i in range(len(shapes))]

            def check(i, form=form):
                m, k, n = shapes[i]
                j0, j1, r = picks[i]
                if form == 0:
                    want = O.matmul_mm_columns(bt.hA[i], bt.hB[i], m, k, n, 8, [j0, j1], threads=1)
                    return bool(O.same_bits(got[i][[j0, j1]], want).all())
                want, _ = O.crt_gemm(bt.hA[i], bt.hB[i], m, k, n, rows=(r, r + 1))
                return bool(O.same_bits(got[i][:, r, :], want.reshape(n, 2)).all())

            ok = O.parallel_map(check, list(range(len(shapes))))
            bad = [i for i, v in enumerate(ok) if not v]
            assert not bad, (form, bad[:10], [shapes[i] for i in bad[:10]])
        finally:
            cuda_lib.mfcuda_batch_destroy(p)


def test_ragged_10k_exp_log_arrays(cuda_lib, dev):
    """Config 4: 10^4 ragged exp / log arrays, lengths log-uniform in [64, 2^20]
    (about 1.1e9 elements, generated on the device), one grouped launch; every
    tenth array is copied back and compared element for element with the oracle."""
    import torch

    rng = np.random.default_rng(10000)
    lens = [int(v) for v in np.exp(rng.uniform(np.log(64), np.log(1 << 20), 10000))]
    offs = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    tot = int(offs[-1])
    g = torch.Generator(device=dev)
    g.manual_seed(11)
    x = torch.empty(2 * tot, dtype=torch.float64, device=dev)
    xv = x.view(-1, 2)
    xv[:, 0].uniform_(-20.0, 20.0, generator=g)  # exp: moderate range; log takes |x|
    xv[:, 1] = xv[:, 0] * (2.0 ** -60)
    y = torch.empty_like(x)
    X = (C.c_void_p * len(lens))(*[x[2 * int(o):].data_ptr() for o in offs[:-1]])
    Y = (C.c_void_p * len(lens))(*[y[2 * int(o):].data_ptr() for o in offs[:-1]])
    N = (C.c_int64 * len(lens))(*lens)
    for op, code in (("exp", 0), ("log", 1)):
        if op == "log":
            xv.abs_()
        p = C.c_void_p()
        assert cuda_lib.mfcuda_batch_create_unary(code, X, Y, N, len(lens), C.byref(p)) == 0
        try:
            y.fill_(float("nan"))
            assert cuda_lib.mfcuda_batch_run(p, _stream()) == 0
            assert cuda_lib.mfcuda_batch_status(p) == 0
            torch.cuda.synchronize()
            sample = list(range(0, len(lens), 10))

            def check(i):
                return bool(O.same_bits(ys[i], O.unary(op, xs[i])).all())

            xs = {i: x[2 * int(offs[i]):2 * int(offs[i + 1])].cpu().numpy() for i in sample}
            ys = {i: y[2 * int(offs[i]):2 * int(offs[i + 1])].cpu().numpy() for i in sample}
            ok = O.parallel_map(check, sample)
            assert all(ok), (op, [sample[q] for q, v in enumerate(ok) if not v][:10])
        finally:
            cuda_lib.mfcuda_batch_destroy(p)
