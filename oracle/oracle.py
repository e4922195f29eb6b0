"""ORACLE -- test infrastructure only (the checker; never part of the product path).

ctypes wrappers around
  * oracle/liboracle.so     the C restatement of the reference algorithms (mf_oracle.c)
  * oracle/_ref/libmfref.so the reference library itself, compiled from its own
                            sources by oracle/Makefile where they are present
All arrays are float64 numpy buffers with interleaved limbs, as in the C ABI.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libmfref.so")

P = C.c_void_p
I64 = C.c_int64
OPS = {"exp": 0, "log": 1, "sin": 2, "cos": 3, "sqrt": 4, "exp2": 5, "log2": 6, "log10": 7}
PAIRS = {"sincos": 0, "cexpi": 1, "cexp": 2}
KINDS = {"sum": 0, "dot": 1, "norm2": 2, "csum": 3, "cdot": 4, "cnorm2": 5}

_orc = None
_ref = None


class _DD(C.Structure):
    _fields_ = [("hi", C.c_double), ("lo", C.c_double)]


def build(ref: bool = False) -> None:
    args = ["make", "-s", "-C", HERE, "oracle"]
    subprocess.run(args, check=True)
    if ref:
        subprocess.run(["make", "-s", "-C", HERE, "ref"], check=True)


def orc():
    global _orc
    if _orc is None:
        src = os.path.join(HERE, "mf_oracle.c")
        if not os.path.exists(ORACLE_SO) or os.path.getmtime(ORACLE_SO) < os.path.getmtime(src):
            build()
        L = C.CDLL(ORACLE_SO)
        L.orc_unary.argtypes = [C.c_int, P, P, I64]
        L.orc_pair.argtypes = [C.c_int, P, P, P, I64]
        L.orc_binary.argtypes = [C.c_int, P, P, P, I64]
        L.orc_matmul_mm.argtypes = [P, P, P, I64, I64, I64, I64]
        L.orc_matmul_mm_block.argtypes = [P, P, P, I64, I64, I64, I64, I64, I64, I64, I64]
        L.orc_matmul_mv.argtypes = [P, P, P, I64, I64, I64]
        L.orc_matmul_vm.argtypes = [P, P, P, I64, I64, I64]
        L.orc_cmatmul_mm.argtypes = [P, P, P, I64, I64, I64, I64]
        for f in ("orc_sum_serial", "orc_csum_serial", "orc_norm2_serial", "orc_cnorm2_serial"):
            getattr(L, f).argtypes = [P, I64, P]
        for f in ("orc_dot_serial", "orc_cdot_serial"):
            getattr(L, f).argtypes = [P, P, I64, I64, P]
        L.orc_reduce_geometry.argtypes = [I64, C.POINTER(I64), C.POINTER(I64)]
        L.orc_reduce_blocked.argtypes = [C.c_int, P, P, I64, I64, P]
        L.orc_reduce_blocked_partial.argtypes = [C.c_int, P, P, I64, I64, P]
        L.orc_reduce_combine.argtypes = [C.c_int, P, I64, P]
        L.orc_gemm_errors.argtypes = [P, P, P, I64, I64, I64, P, P, I64, P, P]
        L.orc_reduce_error.argtypes = [C.c_int, P, P, I64, P, P, P]
        L.orc_split_gemm.argtypes = [P, P, P, I64, I64, I64, C.c_int, C.c_double, P]
        L.orc_split_plan.argtypes = [C.c_int, C.c_double, C.c_int, C.c_int]
        L.orc_split_cgemm.argtypes = [P, P, P, I64, I64, I64, C.c_int, C.c_double, P]
        L.orc_split_gemm_kc.argtypes = [P, P, P, I64, I64, I64, C.c_int, C.c_double, P, I64]
        L.orc_split_cgemm_kc.argtypes = [P, P, P, I64, I64, I64, C.c_int, C.c_double, P, I64]
        L.orc_crt_gemm.argtypes = [P, P, P, I64, I64, I64, C.c_int, C.c_double, P]
        L.orc_crt_cgemm.argtypes = [P, P, P, I64, I64, I64, C.c_int, C.c_double, P]
        L.orc_crt_gemm_rows.argtypes = [P, P, P, I64, I64, I64, C.c_int, C.c_double, P, I64, I64]
        L.orc_crt_bound.argtypes = [C.c_int, C.c_int, C.c_int, I64]
        L.orc_crt_bound.restype = C.c_double
        L.orc_crt_plan.argtypes = [C.c_int, C.c_double, C.c_int, C.c_int, I64, C.POINTER(C.c_int)]
        L.orc_grid_round.argtypes = [C.c_double, C.c_double, C.c_int, C.c_int, C.POINTER(I64)]
        L.orc_wgemm.argtypes = [C.c_char, C.c_char, I64, I64, I64, P, P, I64, P, I64, P, P, I64]
        L.orc_wgemm_info.argtypes = [C.c_char, C.c_char, I64, I64, I64, I64, I64, I64]
        L.orc_wtrsm.argtypes = [C.c_char, C.c_char, C.c_char, C.c_char, I64, I64, P, P, I64, P, I64]
        L.orc_wtrsm_info.argtypes = [C.c_char, C.c_char, C.c_char, C.c_char, I64, I64, I64, I64]
        _orc = L
    return _orc


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref():
    """The reference library (None when it was not built here)."""
    global _ref
    if _ref is None and ref_available():
        L = C.CDLL(REF_SO)
        L.ref_unary_array.argtypes = [C.c_int, P, P, I64]
        L.ref_unary_array_mt.argtypes = [C.c_int, P, P, I64, C.c_int]
        L.ref_binary_array.argtypes = [C.c_int, P, P, P, I64]
        L.ref_pair_array.argtypes = [C.c_int, P, P, P, I64]
        L.matmuldd_mm.argtypes = [P, P, P, I64, I64, I64, I64]
        L.matmuldd_mv.argtypes = [P, P, P, I64, I64, I64]
        L.matmuldd_vm.argtypes = [P, P, P, I64, I64, I64]
        L.ref_matmul_mm_mt.argtypes = [P, P, P, I64, I64, I64, I64, C.c_int]
        L.ref_cmatmul_mm.argtypes = [P, P, P, I64, I64, I64, I64]
        L.ref_norm2_serial.argtypes = [P, I64]
        L.ref_wgemm.argtypes = [C.c_char, C.c_char, I64, I64, I64, P, P, I64, P, I64, P, P, I64]
        L.ref_wtrsm.argtypes = [C.c_char, C.c_char, C.c_char, C.c_char, I64, I64, P, P, I64, P, I64]
        L.ref_wgemm_mt.argtypes = [C.c_char, C.c_char, I64, I64, I64, P, P, I64, P, I64, P, P, I64, C.c_int]
        L.ref_wtrsm_mt.argtypes = [C.c_char, C.c_char, C.c_char, C.c_char, I64, I64, P, P, I64, P, I64,
                                   C.c_int]
        L.ref_norm2_serial.restype = _DD
        _ref = L
    return _ref


def _p(a: np.ndarray) -> int:
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data


def _c(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64).reshape(-1)


# ---- C restatement ------------------------------------------------------------
def pair(kind: str, x):
    """sincos / cexpi / cexp restated (orc_pair): (s, c) for sincos, else the
    complex output."""
    x, n, y0, y1 = _pair_out(kind, x)
    orc().orc_pair(PAIRS[kind], _p(x), _p(y0), _p(y1) if y1.size else None, n)
    return (y0, y1) if kind == "sincos" else y0


def parallel_map(fn, items, threads: int = 0) -> list:
    """[fn(item) for item in items] on a thread pool.  The C restatement keeps
    no global state and ctypes releases the GIL during a call, so oracle calls
    on independent data run in parallel."""
    import concurrent.futures as cf

    threads = threads or os.cpu_count() or 1
    if threads <= 1 or len(items) <= 1:
        return [fn(it) for it in items]
    with cf.ThreadPoolExecutor(max_workers=threads) as ex:
        return list(ex.map(fn, items))


def unary(op: str, x, threads: int = 1) -> np.ndarray:
    """The C restatement of op over an array (element ranges split over
    `threads` threads; 0 = every host core)."""
    x = _c(x)
    y = np.empty_like(x)
    n = x.size // 2
    L = orc()
    threads = threads or os.cpu_count() or 1
    bounds = np.linspace(0, n, max(1, min(threads, n // 4096 + 1)) + 1).astype(np.int64)
    spans = [(int(a), int(b)) for a, b in zip(bounds[:-1], bounds[1:]) if b > a]

    def run(span):
        a, b = span
        L.orc_unary(OPS[op], _p(x) + 16 * a, _p(y) + 16 * a, b - a)

    parallel_map(run, spans, threads)
    return y


def binary(op: int, a, b) -> np.ndarray:
    a, b = _c(a), _c(b)
    y = np.empty_like(a)
    orc().orc_binary(op, _p(a), _p(b), _p(y), a.size // 2)
    return y


def matmul_mm(a, b, m, k, n, ri=8) -> np.ndarray:
    a, b = _c(a), _c(b)
    c = np.empty(2 * m * n)
    orc().orc_matmul_mm(_p(a), _p(b), _p(c), m, k, n, ri)
    return c


def matmul_mm_rows(a, b, m, k, n, ri, rows, threads: int = 0) -> np.ndarray:
    """Rows `rows` of C = A B (row indices): every output runs the same
    sequential MAC over p whatever the shape, so row i of C is the 1 x n
    product of row i of A with B.  Returns len(rows) x n x 2 (one thread per row)."""
    a3, b = _c(a).reshape(k, m, 2), _c(b)
    return np.stack(parallel_map(
        lambda i: matmul_mm(np.ascontiguousarray(a3[:, i, :]), b, 1, k, n, ri).reshape(n, 2), list(rows),
        threads))


def matmul_mm_columns(a, b, m, k, n, ri, cols, threads: int = 0) -> np.ndarray:
    """Columns `cols` of C = A B (column indices): column j of C is the m x 1
    product of A with column j of B.  Returns len(cols) x m x 2 (one thread per column)."""
    a, b3 = _c(a), _c(b).reshape(n, k, 2)
    return np.stack(parallel_map(
        lambda j: matmul_mm(a, np.ascontiguousarray(b3[j]), m, k, 1, ri).reshape(m, 2), list(cols), threads))


def matmul_mm_cols(a, b, m, k, n, ri, j0, j1) -> np.ndarray:
    """Columns [j0, j1) of C only (the others are left uninitialised)."""
    a, b = _c(a), _c(b)
    c = np.zeros(2 * m * n)
    orc().orc_matmul_mm_block(_p(a), _p(b), _p(c), m, k, n, ri, 0, m, j0, j1)
    return c


def matmul_mv(a, x, m, k, ri=8) -> np.ndarray:
    a, x = _c(a), _c(x)
    y = np.empty(2 * m)
    orc().orc_matmul_mv(_p(a), _p(x), _p(y), m, k, ri)
    return y


def matmul_vm(x, b, k, n, ri=8) -> np.ndarray:
    x, b = _c(x), _c(b)
    y = np.empty(2 * n)
    orc().orc_matmul_vm(_p(x), _p(b), _p(y), k, n, ri)
    return y


def cmatmul_mm(a, b, m, k, n, ri=8) -> np.ndarray:
    a, b = _c(a), _c(b)
    c = np.empty(4 * m * n)
    orc().orc_cmatmul_mm(_p(a), _p(b), _p(c), m, k, n, ri)
    return c


def _ch(x: str) -> bytes:
    return x.encode()[:1]


def wgemm(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc):
    """wgemm.f90 restated (orc_wgemm): returns (info, C after the call); the
    input C is not modified."""
    a, b, c = _c(a), _c(b), _c(c).copy()
    al, be = _c(alpha).copy(), _c(beta).copy()
    info = orc().orc_wgemm(_ch(transa), _ch(transb), m, n, k, _p(al), _p(a), lda, _p(b), ldb,
                           _p(be), _p(c), ldc)
    return info, c


def wgemm_info(transa, transb, m, n, k, lda, ldb, ldc) -> int:
    return orc().orc_wgemm_info(_ch(transa), _ch(transb), m, n, k, lda, ldb, ldc)


def wtrsm(side, uplo, transa, diag, m, n, alpha, a, lda, b, ldb):
    """wtrsm.f90 restated (orc_wtrsm): returns (info, B after the call)."""
    a, b = _c(a), _c(b).copy()
    al = _c(alpha).copy()
    info = orc().orc_wtrsm(_ch(side), _ch(uplo), _ch(transa), _ch(diag), m, n, _p(al), _p(a), lda,
                           _p(b), ldb)
    return info, b


def wtrsm_info(side, uplo, transa, diag, m, n, lda, ldb) -> int:
    return orc().orc_wtrsm_info(_ch(side), _ch(uplo), _ch(transa), _ch(diag), m, n, lda, ldb)


def reduce_serial(kind: str, x, y=None, ri=8) -> np.ndarray:
    """The reference's serial Fortran semantics."""
    x = _c(x)
    L = orc()
    cplx = kind.startswith("c")
    n = x.size // (4 if cplx else 2)
    out = np.zeros(4)
    if kind == "sum":
        L.orc_sum_serial(_p(x), n, _p(out))
    elif kind == "csum":
        L.orc_csum_serial(_p(x), n, _p(out))
    elif kind == "norm2":
        L.orc_norm2_serial(_p(x), n, _p(out))
    elif kind == "cnorm2":
        L.orc_cnorm2_serial(_p(x), n, _p(out))
    elif kind == "dot":
        y = _c(y)
        L.orc_dot_serial(_p(x), _p(y), n, ri, _p(out))
    elif kind == "cdot":
        y = _c(y)
        L.orc_cdot_serial(_p(x), _p(y), n, ri, _p(out))
    return out[:4] if kind in ("csum", "cdot") else out[:2]


def reduce_blocked(kind: str, x, y=None, ri=8) -> np.ndarray:
    """The device's fixed blocked order, restated."""
    x = _c(x)
    cplx = kind.startswith("c")
    n = x.size // (4 if cplx else 2)
    yy = _c(y) if y is not None else x
    out = np.zeros(4)
    orc().orc_reduce_blocked(KINDS[kind], _p(x), _p(yy), n, ri, _p(out))
    return out[:4] if kind in ("csum", "cdot") else out[:2]


PARTIAL_VALUES = {"sum": 1, "dot": 1, "norm2": 1, "csum": 2, "cdot": 4, "cnorm2": 1}


def reduce_partial(kind: str, x, y=None, ri=8) -> np.ndarray:
    """The device's per-shard partial (mfcuda_reduce_partial), restated:
    PARTIAL_VALUES[kind] DD values as hi/lo pairs."""
    x = _c(x)
    cplx = kind.startswith("c")
    n = x.size // (4 if cplx else 2)
    yy = _c(y) if y is not None else x
    out = np.zeros(8)
    orc().orc_reduce_blocked_partial(KINDS[kind], _p(x), _p(yy), n, ri, _p(out))
    return out[: 2 * PARTIAL_VALUES[kind]]


def reduce_combine(kind: str, parts) -> np.ndarray:
    """Rank-order fold of gathered partials (mfcuda_reduce_combine), restated."""
    parts = _c(parts)
    count = parts.size // (2 * PARTIAL_VALUES[kind])
    out = np.zeros(4)
    orc().orc_reduce_combine(KINDS[kind], _p(parts), count, _p(out))
    return out[:4] if kind in ("csum", "cdot") else out[:2]


def split_gemm(a, b, m, k, n, slices=0, target=8.0, kc=73 * 128):
    """The split-INT8 algorithm restated on the CPU with K chunks of `kc`
    elements; returns (C, (S, rho_a, rho_b))."""
    a, b = _c(a), _c(b)
    c = np.empty(2 * m * n)
    info = np.zeros(3, dtype=np.int32)
    orc().orc_split_gemm_kc(_p(a), _p(b), _p(c), m, k, n, slices, target, info.ctypes.data, kc)
    return c, tuple(int(v) for v in info)


def split_cgemm(a, b, m, k, n, slices=0, target=8.0, kc=73 * 128):
    """Complex split-INT8 product restated on the CPU (K chunks of `kc` in
    each real product); returns (C, (S, rho_a, rho_b))."""
    a, b = _c(a), _c(b)
    c = np.empty(4 * m * n)
    info = np.zeros(3, dtype=np.int32)
    orc().orc_split_cgemm_kc(_p(a), _p(b), _p(c), m, k, n, slices, target, info.ctypes.data, kc)
    return c, tuple(int(v) for v in info)


def crt_gemm(a, b, m, k, n, bits=0, target=8.0, rows=None):
    """CRT split form restated (orc_crt_gemm): returns (C, info) with info =
    [moduli, rho_a, rho_b, W]; rows=(i0, i1) restricts the output to those rows
    (C is then (i1 - i0) x n, column-major)."""
    a, b = _c(a), _c(b)
    info = np.zeros(4, dtype=np.int32)
    i0, i1 = rows if rows is not None else (0, m)
    c = np.empty(2 * (i1 - i0) * n)
    orc().orc_crt_gemm_rows(_p(a), _p(b), _p(c), m, k, n, bits, target, info.ctypes.data, i0, i1)
    return c, info.tolist()


def crt_cgemm(a, b, m, k, n, bits=0, target=8.0):
    """Complex CRT form restated (orc_crt_cgemm): (C, [moduli, rho_a, rho_b, W])."""
    a, b = _c(a), _c(b)
    info = np.zeros(4, dtype=np.int32)
    c = np.empty(4 * m * n)
    orc().orc_crt_cgemm(_p(a), _p(b), _p(c), m, k, n, bits, target, info.ctypes.data)
    return c, info.tolist()


def crt_plan(bits, target, rho_a, rho_b, k):
    """(W, moduli) the CRT plan picks."""
    nm = C.c_int(0)
    w = orc().orc_crt_plan(bits, target, rho_a, rho_b, k, C.byref(nm))
    return w, nm.value


def crt_bound(W, rho_a, rho_b, k) -> float:
    return orc().orc_crt_bound(W, rho_a, rho_b, k)


def reduce_geometry(n: int) -> tuple[int, int]:
    b, t = I64(), I64()
    orc().orc_reduce_geometry(n, C.byref(b), C.byref(t))
    return b.value, t.value


def gemm_errors(a, b, c, m, k, n, ii, jj):
    """Exact err = C_ij - (AB)_ij and (|A||B|)_ij for the listed outputs."""
    a, b, c = _c(a), _c(b), _c(c)
    ii = np.ascontiguousarray(ii, dtype=np.int64)
    jj = np.ascontiguousarray(jj, dtype=np.int64)
    err = np.empty(ii.size)
    ab = np.empty(ii.size)
    orc().orc_gemm_errors(_p(a), _p(b), _p(c), m, k, n, ii.ctypes.data, jj.ctypes.data, ii.size,
                          _p(err), _p(ab))
    return err, ab


def reduce_error(kind: str, x, y, res):
    """Exact err = res - exact value and the sum of magnitudes, kind 'sum' or 'dot'."""
    x = _c(x)
    yy = _c(y) if y is not None else x
    res = _c(res)
    err, ab = C.c_double(), C.c_double()
    orc().orc_reduce_error(0 if kind == "sum" else 1, _p(x), _p(yy), x.size // 2, _p(res),
                           C.byref(err), C.byref(ab))
    return err.value, ab.value


# ---- the reference itself -------------------------------------------------------
def ref_unary(op: str, x, threads: int = 1) -> np.ndarray:
    x = _c(x)
    y = np.empty_like(x)
    if threads > 1:
        ref().ref_unary_array_mt(OPS[op], _p(x), _p(y), x.size // 2, threads)
    else:
        ref().ref_unary_array(OPS[op], _p(x), _p(y), x.size // 2)
    return y


def _pair_out(kind: str, x):
    x = _c(x)
    n = x.size // (4 if kind == "cexp" else 2)
    y0 = np.empty(2 * n if kind == "sincos" else 4 * n)
    y1 = np.empty(2 * n) if kind == "sincos" else np.empty(0)
    return x, n, y0, y1


def ref_pair(kind: str, x):
    """The reference's sincosdd / cexpidd / cexpdd over an array: (s, c) for
    sincos, else the complex output."""
    x, n, y0, y1 = _pair_out(kind, x)
    ref().ref_pair_array(PAIRS[kind], _p(x), _p(y0), _p(y1) if y1.size else None, n)
    return (y0, y1) if kind == "sincos" else y0


def ref_binary(op: int, a, b) -> np.ndarray:
    a, b = _c(a), _c(b)
    y = np.empty_like(a)
    ref().ref_binary_array(op, _p(a), _p(b), _p(y), a.size // 2)
    return y


def ref_matmul_mm(a, b, m, k, n, ri=8, threads: int = 1) -> np.ndarray:
    a, b = _c(a), _c(b)
    c = np.empty(2 * m * n)
    ref().ref_matmul_mm_mt(_p(a), _p(b), _p(c), m, k, n, ri, threads)
    return c


def ref_cmatmul_mm(a, b, m, k, n, ri=8) -> np.ndarray:
    a, b = _c(a), _c(b)
    c = np.empty(4 * m * n)
    ref().ref_cmatmul_mm(_p(a), _p(b), _p(c), m, k, n, ri)
    return c


def ref_norm2(x) -> np.ndarray:
    x = _c(x)
    r = ref().ref_norm2_serial(_p(x), x.size // 2)
    return np.array([r.hi, r.lo])


def ref_wgemm(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, threads: int = 1) -> np.ndarray:
    """wgemm.f90's loops on the reference's own operators (valid arguments only),
    columns of C sharded over `threads` threads (bit-identical to one thread)."""
    a, b, c = _c(a), _c(b), _c(c).copy()
    al, be = _c(alpha).copy(), _c(beta).copy()
    ta, tb = transa.upper().replace("C", "T"), transb.upper().replace("C", "T")
    ref().ref_wgemm_mt(_ch(ta), _ch(tb), m, n, k, _p(al), _p(a), lda, _p(b), ldb, _p(be), _p(c), ldc, threads)
    return c


def ref_wtrsm(side, uplo, transa, diag, m, n, alpha, a, lda, b, ldb, threads: int = 1) -> np.ndarray:
    """wtrsm.f90's loops on the reference's own operators (valid arguments only),
    independent vectors of B sharded over `threads` threads."""
    a, b = _c(a), _c(b).copy()
    al = _c(alpha).copy()
    t = transa.upper().replace("C", "T")
    ref().ref_wtrsm_mt(_ch(side.upper()), _ch(uplo.upper()), _ch(t), _ch(diag.upper()), m, n, _p(al),
                       _p(a), lda, _p(b), ldb, threads)
    return b


def ref_matmul_mv(a, x, m, k, ri=8) -> np.ndarray:
    a, x = _c(a), _c(x)
    y = np.empty(2 * m)
    ref().matmuldd_mv(_p(a), _p(x), _p(y), m, k, ri)
    return y


def ref_matmul_vm(x, b, k, n, ri=8) -> np.ndarray:
    x, b = _c(x), _c(b)
    y = np.empty(2 * n)
    ref().matmuldd_vm(_p(x), _p(b), _p(y), k, n, ri)
    return y


# ---- comparison helpers -----------------------------------------------------------
def same_bits(a, b) -> np.ndarray:
    """Elementwise bit equality with every NaN treated as one class (per DD value:
    both limbs must match; a NaN hi limb matches any NaN hi limb)."""
    a = _c(a).reshape(-1, 2)
    b = _c(b).reshape(-1, 2)
    eq = (a.view(np.int64) == b.view(np.int64)).all(axis=1)
    nan = np.isnan(a[:, 0]) & np.isnan(b[:, 0])
    return eq | nan
