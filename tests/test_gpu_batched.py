"""GPU parity of the batched ragged launches (grouped kernels in a CUDA graph):
every problem of a batch equals the single call bit for bit, a graph replay
after refilling the inputs recomputes them, and the autotuner's choices are
valid and cached."""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import to_dev, to_host
from multifloats_b200 import _lib
from multifloats_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _shapes(rng, count, lo, hi):
    """log-uniform shapes in [lo, hi], a few degenerate ones mixed in."""
    sh = np.exp(rng.uniform(np.log(lo), np.log(hi), (count, 3))).astype(int)
    sh[0] = (1, 1, 1)
    if count > 3:
        sh[1] = (5, 0, 7)  # k == 0
        sh[2] = (0, 9, 4)  # empty output
    return [tuple(int(v) for v in s) for s in sh]


class Batch:
    def __init__(self, L, dev, shapes, seed, gen):
        self.L, self.dev, self.shapes = L, dev, shapes
        self.A, self.B, self.C, self.hA, self.hB = [], [], [], [], []
        for i, (m, k, n) in enumerate(shapes):
            a, b = gen(m * k, seed + 2 * i), gen(k * n, seed + 2 * i + 1)
            self.hA.append(a)
            self.hB.append(b)
            self.A.append(to_dev(a, dev) if a.size else None)
            self.B.append(to_dev(b, dev) if b.size else None)
            self.C.append(to_dev(np.full(2 * m * n, np.nan), dev) if m * n else None)
        import torch  # noqa: F401

        descs = (_lib.gemm_desc * len(shapes))()
        for i, (m, k, n) in enumerate(shapes):
            descs[i].a = self.A[i].data_ptr() if self.A[i] is not None else None
            descs[i].b = self.B[i].data_ptr() if self.B[i] is not None else None
            descs[i].c = self.C[i].data_ptr() if self.C[i] is not None else None
            descs[i].m, descs[i].k, descs[i].n = m, k, n
        self.descs = descs

    def plan(self, form, ri=8, slices=0, tune=0):
        p = C.c_void_p()
        rc = self.L.mfcuda_batch_create_gemm(self.descs, len(self.shapes), form, ri, slices, 8.0, tune,
                                             C.byref(p))
        assert rc == 0, self.L.mfcuda_error_string(rc)
        return p

    def run(self, p):
        import torch

        assert self.L.mfcuda_batch_run(p, C.c_void_p(torch.cuda.current_stream().cuda_stream)) == 0
        assert self.L.mfcuda_batch_status(p) == 0

    def result(self, i):
        m, k, n = self.shapes[i]
        return to_host(self.C[i]) if m * n else np.zeros(0)


def test_plain_batch_bit_exact(cuda_lib, dev):
    rng = np.random.default_rng(0)
    shapes = _shapes(rng, 40, 1, 200)
    bt = Batch(cuda_lib, dev, shapes, 100, W.dd_uniform)
    p = bt.plan(0, ri=8)
    try:
        edges = {cuda_lib.mfcuda_batch_config(p, i) for i in range(len(shapes))}
        assert edges <= {16, 32, 64} and len(edges) >= 2
        bt.run(p)
        for i, (m, k, n) in enumerate(shapes):
            if m * n == 0:
                continue
            want = O.matmul_mm(bt.hA[i], bt.hB[i], m, k, n, 8)
            assert O.same_bits(bt.result(i), want).all(), (i, m, k, n)
        # replay after refilling the same input buffers
        for i, (m, k, n) in enumerate(shapes):
            if bt.A[i] is not None:
                bt.hA[i] = W.dd_uniform(m * k, 999 + i)
                bt.A[i].copy_(to_dev(bt.hA[i], dev))
        bt.run(p)
        for i, (m, k, n) in enumerate(shapes):
            if m * n:
                assert O.same_bits(bt.result(i), O.matmul_mm(bt.hA[i], bt.hB[i], m, k, n, 8)).all()
    finally:
        cuda_lib.mfcuda_batch_destroy(p)


def test_plain_batch_tuned(cuda_lib, dev):
    rng = np.random.default_rng(1)
    shapes = _shapes(rng, 24, 8, 300)
    bt = Batch(cuda_lib, dev, shapes, 300, W.dd_uniform)
    p = bt.plan(0, ri=5, tune=1)
    try:
        bt.run(p)
        for i, (m, k, n) in enumerate(shapes):
            if m * n:
                assert O.same_bits(bt.result(i), O.matmul_mm(bt.hA[i], bt.hB[i], m, k, n, 5)).all()
    finally:
        cuda_lib.mfcuda_batch_destroy(p)
    path = os.environ["MFCUDA_AUTOTUNE_CACHE"]
    assert os.path.exists(path) and ":plain:" in open(path).read()


@pytest.mark.parametrize("tune", [0, 1])
def test_split_batch_bit_exact(cuda_lib, dev, tune):
    rng = np.random.default_rng(2 + tune)
    shapes = _shapes(rng, 20, 4, 300)
    gen = lambda n, s: W.dd_uniform(n, s)  # noqa: E731
    bt = Batch(cuda_lib, dev, shapes, 500, gen)
    p = bt.plan(1, tune=tune)
    try:
        widths = {cuda_lib.mfcuda_batch_config(p, i) for i in range(len(shapes))}
        assert widths <= {64, 128, 256}
        kc = cuda_lib.mfcuda_batch_kchunk(p)
        assert kc > 0 and kc % 128 == 0
        bt.run(p)
        for i, (m, k, n) in enumerate(shapes):
            if m * n == 0:
                continue
            want, _ = O.split_gemm(bt.hA[i], bt.hB[i], m, k, n, kc=kc)
            assert O.same_bits(bt.result(i), want).all(), (i, m, k, n, kc)
    finally:
        cuda_lib.mfcuda_batch_destroy(p)


def test_split_batch_small_uses_split_k(cuda_lib, dev):
    """A single tall-K product cannot fill the GPU: the plan shortens the K chunk."""
    shapes = [(64, 6000, 40)]
    bt = Batch(cuda_lib, dev, shapes, 700, W.dd_uniform)
    p = bt.plan(1)
    try:
        kc = cuda_lib.mfcuda_batch_kchunk(p)
        assert kc < 73 * 128
        bt.run(p)
        want, _ = O.split_gemm(bt.hA[0], bt.hB[0], 64, 6000, 40, kc=kc)
        assert O.same_bits(bt.result(0), want).all()
    finally:
        cuda_lib.mfcuda_batch_destroy(p)


@pytest.mark.parametrize("op", ["exp", "log", "sin"])
def test_ragged_unary(cuda_lib, dev, op):
    import torch

    rng = np.random.default_rng(5)
    lens = [int(v) for v in np.exp(rng.uniform(np.log(1), np.log(5000), 30))]
    lens[3] = 0
    xs = [W.ELEMENTWISE_INPUTS[op](n, 10 + i) for i, n in enumerate(lens)]
    dx = [to_dev(x, dev) if x.size else torch.empty(0, dtype=torch.float64, device=dev) for x in xs]
    dy = [torch.empty_like(t) for t in dx]
    X = (C.c_void_p * len(lens))(*[t.data_ptr() for t in dx])
    Y = (C.c_void_p * len(lens))(*[t.data_ptr() for t in dy])
    N = (C.c_int64 * len(lens))(*lens)
    code = {"exp": 0, "log": 1, "sin": 2}[op]
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert cuda_lib.mfcuda_unary_dd_ragged(code, X, Y, N, len(lens), stream) == 0
    for x, y in zip(xs, dy):
        assert O.same_bits(to_host(y), O.unary(op, x)).all()
    # the graph form
    for t in dy:
        t.fill_(0.0)
    p = C.c_void_p()
    assert cuda_lib.mfcuda_batch_create_unary(code, X, Y, N, len(lens), C.byref(p)) == 0
    try:
        assert cuda_lib.mfcuda_batch_work_items(p) == sum(lens)
        assert cuda_lib.mfcuda_batch_run(p, stream) == 0
        assert cuda_lib.mfcuda_batch_status(p) == 0
        for x, y in zip(xs, dy):
            assert O.same_bits(to_host(y), O.unary(op, x)).all()
    finally:
        cuda_lib.mfcuda_batch_destroy(p)


def test_batch_invalid_arguments(cuda_lib):
    p = C.c_void_p()
    d = (_lib.gemm_desc * 1)()
    d[0].m, d[0].k, d[0].n = -1, 2, 2
    assert cuda_lib.mfcuda_batch_create_gemm(d, 1, 0, 8, 0, 8.0, 0, C.byref(p)) == 1
    d[0].m = 2
    assert cuda_lib.mfcuda_batch_create_gemm(d, 1, 7, 8, 0, 8.0, 0, C.byref(p)) == 1  # bad form
    assert cuda_lib.mfcuda_batch_create_gemm(d, 1, 2, 8, 5, 8.0, 0, C.byref(p)) == 1  # CRT bits below 8
    assert cuda_lib.mfcuda_batch_create_gemm(d, 1, 2, 8, 111, 8.0, 0, C.byref(p)) == 1  # CRT bits above 110
    assert cuda_lib.mfcuda_batch_create_gemm(d, 1, 0, 8, 0, 8.0, 0, C.byref(p)) == 1  # NULL pointers
    assert cuda_lib.mfcuda_batch_run(None, None) == 1


# ---- complex64x2 batches (the complex configuration's batch of uneven products) ----
class CBatch:
    """Complex problems: A (m x k), B (k x n), C (m x n) complex64x2, column-major."""

    def __init__(self, L, dev, shapes, seed, R=0):
        self.L, self.shapes = L, shapes
        self.A, self.B, self.C, self.hA, self.hB = [], [], [], [], []
        for i, (m, k, n) in enumerate(shapes):
            a = W.complex_from_parts(W.dd_rowcol_scaled(m, k, R, "row", seed + 4 * i) if m * k else np.zeros(0),
                                     W.dd_rowcol_scaled(m, k, R, "row", seed + 4 * i + 1) if m * k else np.zeros(0))
            b = W.complex_from_parts(W.dd_rowcol_scaled(k, n, R, "col", seed + 4 * i + 2) if k * n else np.zeros(0),
                                     W.dd_rowcol_scaled(k, n, R, "col", seed + 4 * i + 3) if k * n else np.zeros(0))
            self.hA.append(a)
            self.hB.append(b)
            self.A.append(to_dev(a, dev) if a.size else None)
            self.B.append(to_dev(b, dev) if b.size else None)
            self.C.append(to_dev(np.full(4 * m * n, np.nan), dev) if m * n else None)
        descs = (_lib.gemm_desc * len(shapes))()
        for i, (m, k, n) in enumerate(shapes):
            descs[i].a = self.A[i].data_ptr() if self.A[i] is not None else None
            descs[i].b = self.B[i].data_ptr() if self.B[i] is not None else None
            descs[i].c = self.C[i].data_ptr() if self.C[i] is not None else None
            descs[i].m, descs[i].k, descs[i].n = m, k, n
        self.descs = descs

    def plan(self, form, ri=8, tune=0):
        p = C.c_void_p()
        rc = self.L.mfcuda_batch_create_cgemm(self.descs, len(self.shapes), form, ri, 0, 8.0, tune, C.byref(p))
        assert rc == 0, self.L.mfcuda_error_string(rc)
        return p

    def run(self, p):
        import torch

        assert self.L.mfcuda_batch_run(p, C.c_void_p(torch.cuda.current_stream().cuda_stream)) == 0
        assert self.L.mfcuda_batch_status(p) == 0


def test_complex_plain_batch_bit_exact(cuda_lib, dev):
    rng = np.random.default_rng(11)
    shapes = _shapes(rng, 30, 1, 160)
    bt = CBatch(cuda_lib, dev, shapes, 900)
    p = bt.plan(0, ri=8)
    try:
        assert {cuda_lib.mfcuda_batch_config(p, i) for i in range(len(shapes))} == {32}
        bt.run(p)
        for i, (m, k, n) in enumerate(shapes):
            if m * n == 0:
                continue
            want = O.cmatmul_mm(bt.hA[i], bt.hB[i], m, k, n, 8)
            assert O.same_bits(to_host(bt.C[i]), want).all(), (i, m, k, n)
    finally:
        cuda_lib.mfcuda_batch_destroy(p)


@pytest.mark.parametrize("tune", [0, 1])
def test_complex_split_batch_bit_exact(cuda_lib, dev, tune):
    rng = np.random.default_rng(12 + tune)
    shapes = _shapes(rng, 14, 4, 260)
    bt = CBatch(cuda_lib, dev, shapes, 1300, R=8)
    p = bt.plan(1, tune=tune)
    try:
        kc = cuda_lib.mfcuda_batch_kchunk(p)
        assert kc > 0 and kc % 128 == 0
        bt.run(p)
        for i, (m, k, n) in enumerate(shapes):
            if m * n == 0:
                continue
            want, _ = O.split_cgemm(bt.hA[i], bt.hB[i], m, k, n, kc=kc)
            assert O.same_bits(to_host(bt.C[i]), want).all(), (i, m, k, n, kc)
    finally:
        cuda_lib.mfcuda_batch_destroy(p)


def test_complex_split_batch_matches_single_call(cuda_lib, dev):
    """With the single call's K chunk the batch reproduces mfcuda_cmatmuldd_mm_split."""
    import torch

    shapes = [(200, 300, 150)] * 40  # enough items that the plan keeps full K chunks
    bt = CBatch(cuda_lib, dev, shapes, 1700, R=16)
    p = bt.plan(1)
    try:
        assert cuda_lib.mfcuda_batch_kchunk(p) == 73 * 128
        bt.run(p)
        m, k, n = shapes[0]
        c = torch.empty(4 * m * n, dtype=torch.float64, device=dev)
        rc = cuda_lib.mfcuda_cmatmuldd_mm_split(bt.A[0].data_ptr(), bt.B[0].data_ptr(), c.data_ptr(), m, k, n, 0,
                                                8.0, None, 0, None,
                                                C.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert rc == 0
        assert O.same_bits(to_host(bt.C[0]), to_host(c)).all()
    finally:
        cuda_lib.mfcuda_batch_destroy(p)


# ---- CRT (modular) split form in the grouped pipeline ----
@pytest.mark.parametrize("tune", [0, 1])
def test_crt_batch_bit_exact(cuda_lib, dev, tune):
    """Every problem equals the CRT restatement bit for bit, whatever K chunk
    the plan chose (residues of chunk sums add modulo each modulus)."""
    rng = np.random.default_rng(40 + tune)
    shapes = _shapes(rng, 20, 4, 300)
    bt = Batch(cuda_lib, dev, shapes, 2100, W.dd_uniform)
    p = bt.plan(2, tune=tune)
    try:
        assert {cuda_lib.mfcuda_batch_config(p, i) for i in range(len(shapes))} <= {64, 128, 256}
        bt.run(p)
        for i, (m, k, n) in enumerate(shapes):
            if m * n == 0:
                continue
            want, _ = O.crt_gemm(bt.hA[i], bt.hB[i], m, k, n)
            assert O.same_bits(bt.result(i), want).all(), (i, m, k, n)
        if tune:
            assert ":crt:" in open(os.environ["MFCUDA_AUTOTUNE_CACHE"]).read()
    finally:
        cuda_lib.mfcuda_batch_destroy(p)


def test_crt_batch_fixed_bits_and_split_k(cuda_lib, dev):
    """A forced operand width, and one tall-K product whose plan shortens the K
    chunk: still the restatement's bits."""
    shapes = [(64, 6000, 40), (130, 700, 33)]
    bt = Batch(cuda_lib, dev, shapes, 2300, W.dd_uniform)
    p = bt.plan(2, slices=64)
    try:
        assert cuda_lib.mfcuda_batch_kchunk(p) < 73 * 128
        bt.run(p)
        for i, (m, k, n) in enumerate(shapes):
            want, info = O.crt_gemm(bt.hA[i], bt.hB[i], m, k, n, bits=64)
            assert info[3] == 64
            assert O.same_bits(bt.result(i), want).all(), (i, m, k, n)
    finally:
        cuda_lib.mfcuda_batch_destroy(p)


def test_crt_batch_matches_single_call(cuda_lib, dev):
    import torch

    shapes = [(300, 500, 200), (129, 257, 65)]
    bt = Batch(cuda_lib, dev, shapes, 2500, W.dd_uniform)
    p = bt.plan(2)
    try:
        bt.run(p)
        for i, (m, k, n) in enumerate(shapes):
            c = torch.empty(2 * m * n, dtype=torch.float64, device=dev)
            rc = cuda_lib.mfcuda_matmuldd_mm_crt(bt.A[i].data_ptr(), bt.B[i].data_ptr(), c.data_ptr(), m, k, n, 0,
                                                 8.0, None, 0, None,
                                                 C.c_void_p(torch.cuda.current_stream().cuda_stream))
            assert rc == 0
            assert O.same_bits(bt.result(i), to_host(c)).all(), i
    finally:
        cuda_lib.mfcuda_batch_destroy(p)


def test_complex_crt_batch_bit_exact(cuda_lib, dev):
    import torch

    rng = np.random.default_rng(44)
    shapes = _shapes(rng, 12, 4, 240)
    bt = CBatch(cuda_lib, dev, shapes, 2700, R=8)
    p = bt.plan(2)
    try:
        bt.run(p)
        for i, (m, k, n) in enumerate(shapes):
            if m * n == 0:
                continue
            want, _ = O.crt_cgemm(bt.hA[i], bt.hB[i], m, k, n)
            assert O.same_bits(to_host(bt.C[i]), want).all(), (i, m, k, n)
        i = max(range(len(shapes)), key=lambda q: shapes[q][0] * shapes[q][1] * shapes[q][2])
        m, k, n = shapes[i]
        c = torch.empty(4 * m * n, dtype=torch.float64, device=dev)
        rc = cuda_lib.mfcuda_cmatmuldd_mm_crt(bt.A[i].data_ptr(), bt.B[i].data_ptr(), c.data_ptr(), m, k, n, 0, 8.0,
                                              None, 0, None, C.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert rc == 0
        assert O.same_bits(to_host(bt.C[i]), to_host(c)).all()
    finally:
        cuda_lib.mfcuda_batch_destroy(p)
