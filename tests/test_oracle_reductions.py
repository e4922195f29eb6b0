"""CPU checks of the reduction oracle: the serial Fortran semantics, the device's
blocked order and the exact superaccumulator agree within the error bounds of
compensated summation, and the blocked geometry matches the library's."""
import numpy as np
import pytest

from multifloats_b200 import workloads as W
from oracle import oracle as O

ULP = 2.0 ** -104


def test_geometry_matches_library(cuda_lib):
    from multifloats_b200 import api

    for n in [0, 1, 255, 4096, 4097, 10 ** 6, 2 ** 26, 2 ** 30]:
        assert api.reduce_geometry(n) == O.reduce_geometry(n)


def test_superaccumulator_exact():
    x = W.dd_uniform(5000, seed=1)
    # sum(x) - sum(x) == 0 exactly: feed x and -x
    both = np.concatenate([x, -x])
    err, ab = O.reduce_error("sum", both, None, np.zeros(2))
    assert err == 0.0 and ab > 0
    # dot of e_i with itself
    a = np.zeros(20)
    a[0::2] = 1.0
    err, _ = O.reduce_error("dot", a, a, np.array([10.0, 0.0]))
    assert err == 0.0


@pytest.mark.parametrize("n", [0, 1, 100, 70000])
def test_sum_dot_bounds(n):
    x = W.dd_uniform(n, seed=n + 1)
    y = W.dd_uniform(n, seed=n + 2)
    for kind, args in (("sum", (x,)), ("dot", (x, y))):
        for fn in (O.reduce_serial, O.reduce_blocked):
            r = fn(kind, *args) if kind == "sum" else fn(kind, *args, ri=8)
            err, ab = O.reduce_error(kind, x, y if kind == "dot" else None, r)
            assert abs(err) <= 16 * ULP * max(ab, 1e-300) + 1e-300, (kind, fn.__name__, err, ab)


@pytest.mark.parametrize("kind", ["norm2", "csum", "cdot", "cnorm2"])
def test_blocked_close_to_serial(kind):
    n = 50000
    x = W.dd_uniform(2 * n if kind.startswith("c") else n, seed=3)
    y = W.dd_uniform(2 * n if kind.startswith("c") else n, seed=4)
    args = (x, y) if "dot" in kind else (x,)
    s = O.reduce_serial(kind, *args)
    b = O.reduce_blocked(kind, *args)
    s2, b2 = s.reshape(-1, 2), b.reshape(-1, 2)
    scale = np.abs(x).sum() * (np.abs(y).max() if "dot" in kind else 1.0)
    for (sh, sl), (bh, bl) in zip(s2, b2):
        diff = (sh - bh) + (sl - bl)
        assert abs(diff) <= 64 * ULP * max(scale, abs(sh)), (kind, diff)


@pytest.mark.parametrize("ri", [0, 1, 3, 8])
def test_blocked_dot_renorm_variants(ri):
    x = W.dd_uniform(9000, seed=11)
    y = W.dd_uniform(9000, seed=12)
    r = O.reduce_blocked("dot", x, y, ri=ri)
    err, ab = O.reduce_error("dot", x, y, r)
    assert abs(err) <= 16 * ULP * ab
