"""GPU parity: elementwise exp/log/sin/cos/sqrt through the C ABI are bit-identical
to the reference (golden vectors) and to the oracle (NaN compared as a class)."""
import numpy as np
import pytest

from conftest import to_dev, to_host
from multifloats_b200 import api
from multifloats_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu
OPS = ["exp", "log", "sin", "cos", "sqrt"]


def _diff_report(x, got, want):
    ok = O.same_bits(got, want)
    bad = np.flatnonzero(~ok)[:5]
    xs = x.reshape(-1, 2)
    return [(xs[i].tolist(), got.reshape(-1, 2)[i].tolist(), want.reshape(-1, 2)[i].tolist()) for i in bad]


@pytest.mark.parametrize("op", OPS)
def test_golden_device(golden, dev, op):
    x, y = golden[f"unary_{op}_x"], golden[f"unary_{op}_y"]
    got = to_host(api.unary(op, to_dev(x, dev)))
    assert O.same_bits(got, y).all(), _diff_report(x, got, y)


@pytest.mark.parametrize("op", OPS)
def test_config_distribution_vs_oracle(dev, op):
    x = W.ELEMENTWISE_INPUTS[op](1 << 20, seed=4242)
    got = to_host(api.unary(op, to_dev(x, dev)))
    want = O.unary(op, x)
    assert O.same_bits(got, want).all(), _diff_report(x, got, want)


@pytest.mark.parametrize("op", ["exp", "sin"])
def test_unaligned_and_inplace(dev, op):
    import torch

    x = W.ELEMENTWISE_INPUTS[op](10001, seed=9)
    want = O.unary(op, x)
    buf = torch.zeros(x.size + 1, dtype=torch.float64, device=dev)
    buf[1:] = torch.from_numpy(x).to(dev)
    view = buf[1:]  # 8-byte aligned only: exercises the scalar-load path
    out = torch.empty(x.size + 1, dtype=torch.float64, device=dev)[1:]
    api.unary(op, view, out=out)
    assert O.same_bits(to_host(out), want).all()
    t = to_dev(x, dev)
    api.unary(op, t, out=t)  # in place
    assert O.same_bits(to_host(t), want).all()


@pytest.mark.parametrize("op", OPS)
def test_host_dropin(op):
    x = W.ELEMENTWISE_INPUTS[op](3333, seed=21)
    got = api.unary(op, x)  # numpy -> expdd_array & co. (host pointers)
    assert O.same_bits(got, O.unary(op, x)).all()


def test_sizes_zero_and_one(dev):
    import torch

    empty = torch.empty(0, dtype=torch.float64, device=dev)
    assert api.exp(empty).numel() == 0
    x = np.array([1.0, 0.0])
    assert O.same_bits(to_host(api.exp(to_dev(x, dev))), O.unary("exp", x)).all()
