"""GPU parity: the plain compensated DD matmul (mm / mv / vm, real and complex)
through the C ABI is bit-identical to the reference (golden vectors) and the
oracle, and within c*k*2^-104*(|A||B|)_ij of the exact product."""
import numpy as np
import pytest

from conftest import to_dev, to_host
from multifloats_b200 import api
from multifloats_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu
ULP = 2.0 ** -104


def test_golden_shapes(golden, dev):
    for idx, (m, k, n, ri) in enumerate(golden["gemm_shapes"]):
        m, k, n, ri = int(m), int(k), int(n), int(ri)
        a, b = golden[f"gemm{idx}_a"], golden[f"gemm{idx}_b"]
        da, db = to_dev(a, dev), to_dev(b, dev)
        c = to_host(api.matmuldd_mm(da, db, m, k, n, ri))
        assert O.same_bits(c, golden[f"gemm{idx}_c"]).all(), ("mm", m, k, n, ri)
        y = to_host(api.matmuldd_mv(da, to_dev(b[: 2 * k], dev), m, k, ri))
        assert O.same_bits(y, golden[f"gemm{idx}_mv"]).all(), ("mv", m, k, ri)
        y = to_host(api.matmuldd_vm(to_dev(a[: 2 * k], dev), db, k, n, ri))
        assert O.same_bits(y, golden[f"gemm{idx}_vm"]).all(), ("vm", k, n, ri)
        if f"cgemm{idx}_a" in golden.files:
            c = to_host(api.cmatmuldd_mm(to_dev(golden[f"cgemm{idx}_a"], dev),
                                         to_dev(golden[f"cgemm{idx}_b"], dev), m, k, n, ri))
            assert O.same_bits(c, golden[f"cgemm{idx}_c"]).all(), ("cmm", m, k, n, ri)


@pytest.mark.parametrize("ri", [8, 0, 5])
def test_gemm_256_cube(dev, ri):
    m = k = n = 256
    a, b = W.dd_uniform(m * k, seed=0), W.dd_uniform(k * n, seed=1)
    c = to_host(api.matmuldd_mm(to_dev(a, dev), to_dev(b, dev), m, k, n, ri))
    assert O.same_bits(c, O.matmul_mm(a, b, m, k, n, ri)).all()
    rng = np.random.default_rng(ri)
    ii, jj = rng.integers(0, m, 200), rng.integers(0, n, 200)
    err, ab = O.gemm_errors(a, b, c, m, k, n, ii, jj)
    # stated bound: |err| <= c * k * 2^-104 * (|A||B|)_ij with c = 1
    assert np.all(np.abs(err) <= k * ULP * ab), np.max(np.abs(err) / (ULP * ab))


def test_gemm_row_major_adapter(dev):
    """Row-major C = A B equals column-major matmuldd_mm(B, A, C, n, k, m)."""
    m, k, n = 37, 50, 29
    a_rm = W.dd_uniform(m * k, seed=3)  # row-major m x k == column-major k x m
    b_rm = W.dd_uniform(k * n, seed=4)
    c = to_host(api.matmuldd_mm(to_dev(b_rm, dev), to_dev(a_rm, dev), n, k, m, 8))
    assert O.same_bits(c, O.matmul_mm(b_rm, a_rm, n, k, m, 8)).all()


def test_gemm_rectangular_odd(dev):
    for (m, k, n, ri) in [(300, 129, 77, 8), (1, 1000, 1, 8), (513, 3, 65, 2), (64, 64, 1, 8)]:
        a, b = W.dd_uniform(m * k, seed=m), W.dd_uniform(k * n, seed=n)
        c = to_host(api.matmuldd_mm(to_dev(a, dev), to_dev(b, dev), m, k, n, ri))
        assert O.same_bits(c, O.matmul_mm(a, b, m, k, n, ri)).all(), (m, k, n, ri)


def test_gemm_unaligned_views(dev):
    import torch

    m, k, n = 70, 33, 45
    a, b = W.dd_uniform(m * k, seed=5), W.dd_uniform(k * n, seed=6)

    def shifted(x):
        buf = torch.zeros(x.size + 1, dtype=torch.float64, device=dev)
        buf[1:] = torch.from_numpy(x).to(dev)
        return buf[1:]

    c = torch.empty(2 * m * n + 1, dtype=torch.float64, device=dev)[1:]
    api.matmuldd_mm(shifted(a), shifted(b), m, k, n, 8, out=c)
    assert O.same_bits(to_host(c), O.matmul_mm(a, b, m, k, n, 8)).all()


def test_gemm_k_zero_and_empty(dev):
    import torch

    c = api.matmuldd_mm(torch.empty(0, dtype=torch.float64, device=dev),
                        torch.empty(0, dtype=torch.float64, device=dev), 4, 0, 3, 8)
    h = to_host(c)
    assert np.all(h == 0.0) and not np.signbit(h).any()


def test_host_dropin_gemm():
    m, k, n = 96, 80, 72
    a, b = W.dd_uniform(m * k, seed=7), W.dd_uniform(k * n, seed=8)
    c = api.matmuldd_mm(a, b, m, k, n, 8)  # numpy -> matmuldd_mm (host pointers)
    assert O.same_bits(c, O.matmul_mm(a, b, m, k, n, 8)).all()
    y = api.matmuldd_mv(a, b[: 2 * k], m, k, 8)
    assert O.same_bits(y, O.matmul_mv(a, b[: 2 * k], m, k, 8)).all()
    ca = W.complex_from_parts(a, W.dd_uniform(m * k, seed=9))
    cb = W.complex_from_parts(b, W.dd_uniform(k * n, seed=10))
    cc = api.cmatmuldd_mm(ca, cb, m, k, n, 8)
    assert O.same_bits(cc, O.cmatmul_mm(ca, cb, m, k, n, 8)).all()


def test_complex_gemm_larger(dev):
    m, k, n = 130, 70, 66
    ca = W.complex_from_parts(W.dd_uniform(m * k, seed=11), W.dd_uniform(m * k, seed=12))
    cb = W.complex_from_parts(W.dd_uniform(k * n, seed=13), W.dd_uniform(k * n, seed=14))
    c = to_host(api.cmatmuldd_mm(to_dev(ca, dev), to_dev(cb, dev), m, k, n, 8))
    assert O.same_bits(c, O.cmatmul_mm(ca, cb, m, k, n, 8)).all()


def test_gemm_nonfinite_propagates(dev):
    m = k = n = 16
    a, b = W.dd_uniform(m * k, seed=15), W.dd_uniform(k * n, seed=16)
    a[2 * 5] = np.nan
    a[2 * 40] = np.inf
    c = to_host(api.matmuldd_mm(to_dev(a, dev), to_dev(b, dev), m, k, n, 8))
    assert O.same_bits(c, O.matmul_mm(a, b, m, k, n, 8)).all()


def test_mv_vm_large(dev):
    m, k = 3000, 700
    a, x = W.dd_uniform(m * k, seed=17), W.dd_uniform(k, seed=18)
    y = to_host(api.matmuldd_mv(to_dev(a, dev), to_dev(x, dev), m, k, 8))
    assert O.same_bits(y, O.matmul_mv(a, x, m, k, 8)).all()
    xv = W.dd_uniform(m, seed=19)
    y = to_host(api.matmuldd_vm(to_dev(xv, dev), to_dev(a, dev), m, k, 8))
    assert O.same_bits(y, O.matmul_vm(xv, a, m, k, 8)).all()


@pytest.mark.parametrize("ri", [0, 3, 8])
@pytest.mark.parametrize("m,k", [(1, 1), (77, 45), (33, 65), (1000, 97)])
def test_mv_vm_ragged_and_unaligned(dev, m, k, ri):
    """Sizes off the 32-row / 32-k staging grid, every renorm cadence, and
    8-byte-offset (not 16-byte-aligned) operand views."""
    import torch

    a, x, xv = W.dd_uniform(m * k, seed=m + k), W.dd_uniform(k, seed=m + 1), W.dd_uniform(m, seed=k + 2)
    want_mv, want_vm = O.matmul_mv(a, x, m, k, ri), O.matmul_vm(xv, a, m, k, ri)
    for offset in (0, 1):
        def view(v):
            buf = torch.empty(v.size + offset, dtype=torch.float64, device=dev)
            buf[offset:] = torch.from_numpy(v).to(dev)
            return buf[offset:]

        y = to_host(api.matmuldd_mv(view(a), view(x), m, k, ri))
        assert O.same_bits(y, want_mv).all(), ("mv", offset)
        y = to_host(api.matmuldd_vm(view(xv), view(a), m, k, ri))
        assert O.same_bits(y, want_vm).all(), ("vm", offset)
