"""BLAS-style shims: argument checking through the C ABI (no device work is
done on an invalid call, so these run without a GPU).  The info codes follow
test/integration/blas/wgemm.f90:29-48 and wtrsm.f90:24-44."""
import pytest

from multifloats_b200 import api
from oracle import oracle as O


@pytest.mark.parametrize("args", [
    ("X", "N", 2, 3, 4, 2, 4, 2), ("n", "Q", 2, 3, 4, 2, 4, 2), ("T", "N", -1, 3, 4, 4, 4, 1),
    ("N", "N", 2, -3, 4, 2, 4, 2), ("N", "C", 2, 3, -4, 2, 3, 2), ("N", "N", 2, 3, 4, 1, 4, 2),
    ("T", "N", 2, 3, 4, 3, 4, 2), ("N", "N", 2, 3, 4, 2, 3, 2), ("N", "T", 2, 3, 4, 2, 2, 2),
    ("N", "N", 2, 3, 4, 2, 4, 1), ("N", "N", 0, 0, 0, 0, 1, 1),
])
def test_wgemm_info_matches_oracle(args):
    ta, tb, m, n, k, lda, ldb, ldc = args
    want = O.wgemm_info(ta, tb, m, n, k, lda, ldb, ldc)
    assert want != 0
    with pytest.raises(api.BlasArgumentError) as e:
        api.wgemm(ta, tb, m, n, k, 1.0, None, lda, None, ldb, 0.0, None, ldc)
    assert e.value.info == want


@pytest.mark.parametrize("args", [
    ("X", "U", "N", "N", 3, 2, 3, 3), ("r", "X", "N", "N", 3, 2, 3, 3), ("L", "l", "X", "N", 3, 2, 3, 3),
    ("L", "U", "c", "X", 3, 2, 3, 3), ("L", "U", "N", "u", -3, 2, 3, 3), ("L", "U", "N", "N", 3, -2, 3, 3),
    ("L", "U", "N", "N", 3, 2, 2, 3), ("R", "U", "N", "N", 3, 4, 3, 3), ("L", "U", "N", "N", 3, 2, 3, 2),
])
def test_wtrsm_info_matches_oracle(args):
    side, uplo, ta, diag, m, n, lda, ldb = args
    want = O.wtrsm_info(side, uplo, ta, diag, m, n, lda, ldb)
    assert want != 0
    with pytest.raises(api.BlasArgumentError) as e:
        api.wtrsm(side, uplo, ta, diag, m, n, 1.0, None, lda, None, ldb)
    assert e.value.info == want


def test_quick_returns_need_no_device():
    """m = 0 or n = 0 returns before any device work (wgemm.f90:49, wtrsm.f90:45)."""
    assert api.wgemm("N", "N", 0, 5, 3, 1.0, None, 1, None, 3, 0.0, None, 1) is None
    assert api.wtrsm("R", "L", "T", "U", 4, 0, 2.0, None, 1, None, 4) is None
