"""GPU parity: the BLAS-style shims wgemm / wtrsm (DGEMM / DTRSM semantics over
DD matrices, test/integration/blas/wgemm.f90 and wtrsm.f90) through the C ABI
are bit-identical to the reference (golden vectors made with the reference's
operators) and to the oracle on fresh inputs -- both transpositions, padded
leading dimensions, alpha / beta special values, zero and non-finite entries,
several diagonal blocks and vector groups; padding rows are left untouched."""
import numpy as np
import pytest

from conftest import to_dev, to_host, wgemm_golden, wtrsm_golden
from multifloats_b200 import api
from multifloats_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _dev_args_wgemm(args, dev):
    ta, tb, m, n, k, al, a, lda, b, ldb, be, c, ldc = args
    return (ta, tb, m, n, k, al, to_dev(a, dev), lda, to_dev(b, dev), ldb, be, to_dev(c, dev), ldc)


def test_wgemm_golden_device(golden, dev):
    for i, args, want in wgemm_golden(golden):
        d = _dev_args_wgemm(args, dev)
        api.wgemm(*d)
        got = to_host(d[11])
        assert O.same_bits(got, want).all(), (i, args[:5])


def test_wgemm_golden_host(golden):
    for i, args, want in wgemm_golden(golden):
        args = list(args)
        args[11] = args[11].copy()
        api.wgemm(*args)
        assert O.same_bits(args[11], want).all(), (i, args[:5])


def test_wtrsm_golden_device_and_host(golden, dev):
    for i, args, want in wtrsm_golden(golden):
        side, uplo, ta, diag, m, n, al, a, lda, b, ldb = args
        db = to_dev(b, dev)
        api.wtrsm(side, uplo, ta, diag, m, n, al, to_dev(a, dev), lda, db, ldb)
        assert O.same_bits(to_host(db), want).all(), (i, args[:6])
        hb = b.copy()
        api.wtrsm(side, uplo, ta, diag, m, n, al, a, lda, hb, ldb)
        assert O.same_bits(hb, want).all(), (i, args[:6])


def _wgemm_case(ta, tb, m, n, k, pad, seed):
    nota, notb = ta == "N", tb == "N"
    ra, ca = (m, k) if nota else (k, m)
    rb, cb = (k, n) if notb else (n, k)
    lda, ldb, ldc = ra + pad, rb + pad, m + pad
    return (W.dd_padded(ra, ca, lda, seed, zeros=0.05), lda, W.dd_padded(rb, cb, ldb, seed + 1), ldb,
            W.dd_padded(m, n, ldc, seed + 2), ldc)


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("N", "T"), ("T", "N"), ("C", "C")])
@pytest.mark.parametrize("beta", [(0.0, 0.0), (1.0, 0.0), (-0.75, 1e-18)])
def test_wgemm_fresh_vs_oracle(dev, ta, tb, beta):
    rng = np.random.default_rng(hash((ta, tb, beta[0])) % 2**32)
    for (m, n, k, pad) in [(130, 70, 200, 3), (64, 64, 64, 0), (1, 300, 77, 1), (257, 3, 129, 2)]:
        a, lda, b, ldb, c, ldc = _wgemm_case(ta, tb, m, n, k, pad, int(rng.integers(1 << 30)))
        alpha = W.with_lo(rng.uniform(-2, 2, 1), rng)
        info, want = O.wgemm(ta, tb, m, n, k, alpha, a, lda, b, ldb, np.array(beta), c, ldc)
        assert info == 0
        dc = to_dev(c, dev)
        api.wgemm(ta, tb, m, n, k, alpha, to_dev(a, dev), lda, to_dev(b, dev), ldb, beta, dc, ldc)
        got = to_host(dc)
        ok = O.same_bits(got, want)
        assert ok.all(), (m, n, k, np.flatnonzero(~ok)[:5])


def test_wgemm_unaligned_views(dev):
    """8-byte-aligned operands take the scalar-load path; same bits."""
    import torch

    m, n, k = 70, 45, 90
    for ta, tb in [("N", "N"), ("T", "T")]:
        a, lda, b, ldb, c, ldc = _wgemm_case(ta, tb, m, n, k, 1, 31)
        alpha, beta = np.array([1.5, 1e-17]), np.array([0.5, 0.0])
        _, want = O.wgemm(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)

        def shifted(x):
            buf = torch.zeros(x.size + 1, dtype=torch.float64, device=dev)
            buf[1:] = torch.from_numpy(x).to(dev)
            return buf[1:]

        dc = shifted(c)
        api.wgemm(ta, tb, m, n, k, alpha, shifted(a), lda, shifted(b), ldb, beta, dc, ldc)
        assert O.same_bits(to_host(dc), want).all()


@pytest.mark.parametrize("side", ["L", "R"])
@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("ta", ["N", "T"])
@pytest.mark.parametrize("diag", ["N", "U"])
def test_wtrsm_fresh_vs_oracle(dev, side, uplo, ta, diag):
    """Orders spanning several 32-pivot blocks and 64-element chunks, vector
    counts that leave a partial 16-vector group, zero entries that exercise the
    skipped updates."""
    rng = np.random.default_rng(len(side + uplo + ta + diag) * 7 + ord(side) + 3 * ord(uplo) + 5 * ord(ta))
    for (m, n, zeros) in [(100, 37, 0.3), (37, 100, 0.0), (161, 20, 0.1)]:
        na = m if side == "L" else n
        lda, ldb = na + int(rng.integers(0, 3)), m + int(rng.integers(0, 3))
        a = W.dd_triangular(na, lda, int(rng.integers(1 << 30)), zeros=zeros)
        b = W.dd_padded(m, n, ldb, int(rng.integers(1 << 30)), zeros=zeros)
        for alpha in (np.array([1.0, 0.0]), W.with_lo(rng.uniform(-2, 2, 1), rng)):
            info, want = O.wtrsm(side, uplo, ta, diag, m, n, alpha, a, lda, b, ldb)
            assert info == 0
            db = to_dev(b, dev)
            api.wtrsm(side, uplo, ta, diag, m, n, alpha, to_dev(a, dev), lda, db, ldb)
            ok = O.same_bits(to_host(db), want)
            assert ok.all(), (m, n, alpha, np.flatnonzero(~ok)[:5])


def test_wgemm_large_matches_oracle_sample(dev):
    """A 512 x 384 x 640 product (8 x 6 tiles of 64, 80 k-slices): rows sampled
    against the oracle's restatement (the full product is too slow on the CPU)."""
    m, n, k = 512, 384, 640
    a, lda, b, ldb, c, ldc = _wgemm_case("N", "N", m, n, k, 0, 77)
    alpha, beta = np.array([0.75, 0.0]), np.array([-1.25, 3e-17])
    dc = to_dev(c, dev)
    api.wgemm("N", "N", m, n, k, alpha, to_dev(a, dev), lda, to_dev(b, dev), ldb, beta, dc, ldc)
    got = to_host(dc).reshape(n, m, 2)
    rows = [0, 1, 63, 64, 200, 511]
    a3 = a.reshape(k, m, 2)
    sub_a = np.ascontiguousarray(a3[:, rows, :]).reshape(-1)
    sub_c = np.ascontiguousarray(c.reshape(n, m, 2)[:, rows, :]).reshape(-1)
    _, want = O.wgemm("N", "N", len(rows), n, k, alpha, sub_a, len(rows), b, ldb, beta, sub_c, len(rows))
    assert O.same_bits(np.ascontiguousarray(got[:, rows, :]).reshape(-1), want).all()
