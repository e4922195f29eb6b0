"""GPU parity: the sum / dot_product / norm2 reductions (real and complex) through
the C ABI are bit-identical to the CPU restatement of the device's fixed order,
reproducible run to run, and within the compensated-summation bound of the
reference's serial Fortran result and of the exact value."""
import numpy as np
import pytest

from conftest import to_dev, to_host
from multifloats_b200 import api
from multifloats_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu
ULP = 2.0 ** -104
SIZES = [0, 1, 255, 4096 * 16 + 3, (1 << 20) + 7]


def _dev_reduce(kind, x, y, dev, ri=8):
    dx = to_dev(x, dev)
    dy = to_dev(y, dev) if y is not None else None
    fn = {"sum": lambda: api.sum_dd(dx), "dot": lambda: api.dot_product(dx, dy, ri),
          "norm2": lambda: api.norm2(dx), "csum": lambda: api.csum_dd(dx),
          "cdot": lambda: api.cdot_product(dx, dy, ri), "cnorm2": lambda: api.cnorm2(dx)}[kind]
    return to_host(fn())


@pytest.mark.parametrize("kind", ["sum", "dot", "norm2", "csum", "cdot", "cnorm2"])
@pytest.mark.parametrize("n", SIZES)
def test_bit_exact_vs_blocked_order(dev, kind, n):
    cplx = kind.startswith("c")
    x = W.dd_uniform(2 * n if cplx else n, seed=n + 31)
    y = W.dd_uniform(2 * n if cplx else n, seed=n + 32) if "dot" in kind else None
    got = _dev_reduce(kind, x, y, dev)
    want = O.reduce_blocked(kind, x, y, ri=8)
    assert O.same_bits(got, want).all(), (got, want)
    again = _dev_reduce(kind, x, y, dev)
    assert O.same_bits(got, again).all()


@pytest.mark.parametrize("ri", [0, 1, 3, 8, 13])
def test_dot_renorm_intervals(dev, ri):
    n = 300001
    x, y = W.dd_uniform(n, seed=1), W.dd_uniform(n, seed=2)
    got = _dev_reduce("dot", x, y, dev, ri)
    assert O.same_bits(got, O.reduce_blocked("dot", x, y, ri=ri)).all()


@pytest.mark.parametrize("kind", ["sum", "dot"])
def test_within_bound_of_serial_and_exact(dev, kind):
    n = 1 << 22
    x, y = W.dd_uniform(n, seed=3), W.dd_uniform(n, seed=4)
    got = _dev_reduce(kind, x, y if kind == "dot" else None, dev)
    err, ab = O.reduce_error(kind, x, y if kind == "dot" else None, got)
    assert abs(err) <= 16 * ULP * ab, err / (ULP * ab)
    ser = O.reduce_serial(kind, x, y if kind == "dot" else None)
    serr, _ = O.reduce_error(kind, x, y if kind == "dot" else None, ser)
    assert abs(err - serr) <= 32 * ULP * ab


def test_norm2_golden(golden, dev):
    for idx in range(5):
        x = golden[f"norm2_{idx}_x"]
        want = golden[f"norm2_{idx}_y"]
        got = _dev_reduce("norm2", x, None, dev)
        d = abs((got[0] - want[0]) + (got[1] - want[1]))
        assert d <= 64 * ULP * max(abs(want[0]), 1e-300), (idx, got, want)


def test_host_dropin_reductions():
    n = 100003
    x, y = W.dd_uniform(n, seed=5), W.dd_uniform(n, seed=6)
    assert O.same_bits(np.array(api.sum_dd(x)), O.reduce_blocked("sum", x)).all()
    assert O.same_bits(np.array(api.dot_product(x, y, 8)), O.reduce_blocked("dot", x, y, 8)).all()
    assert O.same_bits(np.array(api.norm2(x)), O.reduce_blocked("norm2", x)).all()
    cx = W.complex_from_parts(x, y)
    assert O.same_bits(np.array(api.csum_dd(cx)), O.reduce_blocked("csum", cx)).all()
    assert O.same_bits(np.array(api.cdot_product(cx, cx, 8)), O.reduce_blocked("cdot", cx, cx, 8)).all()
    assert O.same_bits(np.array(api.cnorm2(cx)), O.reduce_blocked("cnorm2", cx)).all()


def test_nonfinite_inputs(dev):
    x = W.dd_uniform(5000, seed=7)
    x[2 * 17] = np.inf
    got = _dev_reduce("sum", x, None, dev)
    assert O.same_bits(got, O.reduce_blocked("sum", x)).all()
    x[2 * 99] = np.nan
    got = _dev_reduce("norm2", x, None, dev)
    assert np.isnan(got[0])


@pytest.mark.parametrize("kind", ["sum", "dot", "norm2", "csum", "cdot", "cnorm2"])
def test_shard_partials_and_rank_combine(dev, kind):
    """mfcuda_reduce_partial over shards, then mfcuda_reduce_combine in shard
    order: bit-identical to the CPU restatement of the same order; one shard
    reproduces the single call."""
    import torch

    from multifloats_b200 import dist as D

    cplx = kind.startswith("c")
    e = 4 if cplx else 2
    n = 3 * 4096 * 5 + 17
    x = W.dd_uniform(2 * n if cplx else n, seed=71)
    y = W.dd_uniform(2 * n if cplx else n, seed=72) if "dot" in kind else None
    be = D.CudaBackend()
    for world in (1, 3, 4):
        parts_dev, parts_cpu = [], []
        for r in range(world):
            a, b = D.shard_bounds(n, r, world)
            xl = to_dev(x[e * a: e * b], dev)
            yl = to_dev(y[e * a: e * b], dev) if y is not None else None
            parts_dev.append(be.partial(kind, xl, yl, 8))
            parts_cpu.append(O.reduce_partial(kind, x[e * a: e * b], y[e * a: e * b] if y is not None else None, 8))
        got = to_host(be.combine(kind, torch.cat(parts_dev)))
        assert O.same_bits(to_host(torch.cat(parts_dev)), np.concatenate(parts_cpu)).all()
        want = O.reduce_combine(kind, np.concatenate(parts_cpu))
        assert O.same_bits(got, want).all(), (world, got, want)
        if world == 1:
            assert O.same_bits(got, O.reduce_blocked(kind, x, y, ri=8)).all()
