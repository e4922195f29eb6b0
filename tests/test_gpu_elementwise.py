"""GPU parity: elementwise exp/log/sin/cos/sqrt/exp2/log2/log10 and the fused
sincos / cexpi / cexp maps through the C ABI are bit-identical to the reference
(golden vectors) and to the oracle (NaN compared as a class)."""
import numpy as np
import pytest

from conftest import to_dev, to_host
from multifloats_b200 import api
from multifloats_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu
OPS = ["exp", "log", "sin", "cos", "sqrt", "exp2", "log2", "log10"]
INPUTS = {**W.ELEMENTWISE_INPUTS, **W.EXTRA_ELEMENTWISE_INPUTS}


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
    x = INPUTS[op](1 << 20, seed=4242)
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
    x = INPUTS[op](3333, seed=21)
    got = api.unary(op, x)  # numpy -> expdd_array & co. (host pointers)
    assert O.same_bits(got, O.unary(op, x)).all()


def test_sizes_zero_and_one(dev):
    import torch

    empty = torch.empty(0, dtype=torch.float64, device=dev)
    assert api.exp(empty).numel() == 0
    x = np.array([1.0, 0.0])
    assert O.same_bits(to_host(api.exp(to_dev(x, dev))), O.unary("exp", x)).all()


def test_sincos_cexpi_cexp_golden_device(golden, dev):
    x = golden["pair_sincos_x"]
    s, c = api.sincos(to_dev(x, dev))
    assert O.same_bits(to_host(s), golden["pair_sincos_s"]).all(), _diff_report(x, to_host(s), golden["pair_sincos_s"])
    assert O.same_bits(to_host(c), golden["pair_sincos_c"]).all(), _diff_report(x, to_host(c), golden["pair_sincos_c"])
    z = to_host(api.cexpi(to_dev(golden["pair_cexpi_x"], dev)))
    assert O.same_bits(z, golden["pair_cexpi_z"]).all()
    w = to_host(api.cexp(to_dev(golden["pair_cexp_x"], dev)))
    ok = O.same_bits(w, golden["pair_cexp_w"])
    assert ok.all(), (np.count_nonzero(~ok), np.flatnonzero(~ok)[:8])


def test_sincos_cexp_distribution_unaligned_and_host(dev):
    import torch

    x = W.ELEMENTWISE_INPUTS["sin"](100003, seed=31)
    ws, wc = O.pair("sincos", x)
    buf = torch.zeros(x.size + 1, dtype=torch.float64, device=dev)
    buf[1:] = torch.from_numpy(x).to(dev)
    s = torch.empty(x.size + 1, dtype=torch.float64, device=dev)[1:]
    c = torch.empty(x.size + 1, dtype=torch.float64, device=dev)[1:]
    api.sincos(buf[1:], s, c)  # 8-byte-aligned views: the scalar-load path
    assert O.same_bits(to_host(s), ws).all() and O.same_bits(to_host(c), wc).all()
    # equal to the separate sine and cosine kernels
    assert O.same_bits(to_host(s), to_host(api.unary("sin", to_dev(x, dev)))).all()
    assert O.same_bits(to_host(c), to_host(api.unary("cos", to_dev(x, dev)))).all()
    hs, hc = api.sincos(x)  # host drop-in
    assert O.same_bits(hs, ws).all() and O.same_bits(hc, wc).all()
    rng = np.random.default_rng(32)
    z = W.complex_from_parts(W.with_lo(rng.uniform(-700.0, 700.0, 50001), rng),
                             W.ELEMENTWISE_INPUTS["sin"](50001, seed=33))
    want = O.pair("cexp", z)
    assert O.same_bits(to_host(api.cexp(to_dev(z, dev))), want).all()
    assert O.same_bits(api.cexp(z), want).all()
    assert O.same_bits(api.cexpi(x), O.pair("cexpi", x)).all()
