"""Python mirror of the libmultifloats_cuda C ABI.

Arrays are float64 buffers whose trailing axis holds the limbs: a float64x2
array of n elements is any float64 array with 2n entries (hi, lo interleaved),
a complex64x2 array has 4n entries (re.hi, re.lo, im.hi, im.lo).  Matrices are
column-major with leading dimension = number of rows, exactly as in the C ABI
(and in the reference's matmuldd_* functions).

Every function accepts either host numpy arrays -- routed through the drop-in
symbols (host pointers, synchronous) -- or CUDA torch tensors, routed through
the mfcuda_* device API on torch's current stream.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, check_last, complex64x2, float64x2, lib

OP = {"exp": 0, "log": 1, "sin": 2, "cos": 3, "sqrt": 4, "exp2": 5, "log2": 6, "log10": 7}


def _is_dev(x) -> bool:
    return hasattr(x, "is_cuda") and bool(x.is_cuda)


def _ptr(x) -> int:
    if x is None:
        return 0
    if _is_dev(x):
        return x.data_ptr()
    return x.ctypes.data


def _stream():
    import torch

    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _host(x, n_doubles: int, name: str) -> np.ndarray:
    a = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
    if a.size != n_doubles:
        raise ValueError(f"{name}: expected {n_doubles} doubles, got {a.size}")
    return a


def _dev_check(x, n_doubles: int, name: str):
    """A device call's operand must be a contiguous float64 CUDA tensor: a host
    pointer handed to a kernel would fault, so mixed host / device operands
    are refused here."""
    import torch

    if (not _is_dev(x) or x.dtype != torch.float64 or not x.is_contiguous() or x.numel() != n_doubles):
        raise ValueError(f"{name}: expected a contiguous float64 CUDA tensor of {n_doubles} doubles")
    return x


def _host_out(x, n_doubles: int, name: str) -> np.ndarray:
    """A caller-supplied host output must be written in place: a C-contiguous
    float64 numpy array of exactly n_doubles entries."""
    if not (isinstance(x, np.ndarray) and x.dtype == np.float64 and x.flags.c_contiguous and x.size == n_doubles):
        raise ValueError(f"{name}: expected a C-contiguous float64 numpy array of {n_doubles} doubles")
    return x


def _empty_like_kind(ref, n_doubles: int):
    if _is_dev(ref):
        import torch

        return torch.empty(n_doubles, dtype=torch.float64, device=ref.device)
    return np.empty(n_doubles, dtype=np.float64)


# ---- matmul ------------------------------------------------------------------
def matmuldd_mm(a, b, m: int, k: int, n: int, renorm_interval: int = 8, out=None):
    """C(m,n) = A(m,k) B(k,n), column-major DD (reference matmuldd_mm)."""
    L = lib()
    if _is_dev(a):
        a, b = _dev_check(a, 2 * m * k, "a"), _dev_check(b, 2 * k * n, "b")
        c = _dev_check(out, 2 * m * n, "out") if out is not None else _empty_like_kind(a, 2 * m * n)
        check(L.mfcuda_matmuldd_mm(_ptr(a), _ptr(b), _ptr(c), m, k, n, renorm_interval, _stream()),
              "mfcuda_matmuldd_mm")
        return c
    a, b = _host(a, 2 * m * k, "a"), _host(b, 2 * k * n, "b")
    c = _host_out(out, 2 * m * n, "out") if out is not None else np.empty(2 * m * n)
    L.matmuldd_mm(_ptr(a), _ptr(b), _ptr(c), m, k, n, renorm_interval)
    check_last("matmuldd_mm")
    return c


def matmuldd_mv(a, x, m: int, k: int, renorm_interval: int = 8):
    L = lib()
    if _is_dev(a):
        y = _empty_like_kind(a, 2 * m)
        check(L.mfcuda_matmuldd_mv(_ptr(_dev_check(a, 2 * m * k, "a")), _ptr(_dev_check(x, 2 * k, "x")),
                                   _ptr(y), m, k, renorm_interval, _stream()), "mfcuda_matmuldd_mv")
        return y
    a, x = _host(a, 2 * m * k, "a"), _host(x, 2 * k, "x")
    y = np.empty(2 * m)
    L.matmuldd_mv(_ptr(a), _ptr(x), _ptr(y), m, k, renorm_interval)
    check_last("matmuldd_mv")
    return y


def matmuldd_vm(x, b, k: int, n: int, renorm_interval: int = 8):
    L = lib()
    if _is_dev(b):
        y = _empty_like_kind(b, 2 * n)
        check(L.mfcuda_matmuldd_vm(_ptr(_dev_check(x, 2 * k, "x")), _ptr(_dev_check(b, 2 * k * n, "b")),
                                   _ptr(y), k, n, renorm_interval, _stream()), "mfcuda_matmuldd_vm")
        return y
    x, b = _host(x, 2 * k, "x"), _host(b, 2 * k * n, "b")
    y = np.empty(2 * n)
    L.matmuldd_vm(_ptr(x), _ptr(b), _ptr(y), k, n, renorm_interval)
    check_last("matmuldd_vm")
    return y


def cmatmuldd_mm(a, b, m: int, k: int, n: int, renorm_interval: int = 8, out=None):
    """Complex C = A B as the Fortran cdd_matmul_mm composition (4 real products)."""
    L = lib()
    if _is_dev(a):
        a, b = _dev_check(a, 4 * m * k, "a"), _dev_check(b, 4 * k * n, "b")
        c = _dev_check(out, 4 * m * n, "out") if out is not None else _empty_like_kind(a, 4 * m * n)
        check(L.mfcuda_cmatmuldd_mm(_ptr(a), _ptr(b), _ptr(c), m, k, n, renorm_interval, _stream()),
              "mfcuda_cmatmuldd_mm")
        return c
    a, b = _host(a, 4 * m * k, "a"), _host(b, 4 * k * n, "b")
    c = _host_out(out, 4 * m * n, "out") if out is not None else np.empty(4 * m * n)
    L.cmatmuldd_mm(_ptr(a), _ptr(b), _ptr(c), m, k, n, renorm_interval)
    check_last("cmatmuldd_mm")
    return c


# ---- split-INT8 forms (no reference counterpart) --------------------------------------
_SPLIT_SYMS = {("split", False): ("mfcuda_matmuldd_mm_split", "matmuldd_mm_split"),
               ("split", True): ("mfcuda_cmatmuldd_mm_split", "cmatmuldd_mm_split"),
               ("crt", False): ("mfcuda_matmuldd_mm_crt", "matmuldd_mm_crt"),
               ("crt", True): ("mfcuda_cmatmuldd_mm_crt", "cmatmuldd_mm_crt")}


def _split_call(form: str, cplx: bool, a, b, m: int, k: int, n: int, arg: int, target: float, out):
    L = lib()
    w = 4 if cplx else 2
    dev_sym, host_sym = _SPLIT_SYMS[(form, cplx)]
    if _is_dev(a):
        a, b = _dev_check(a, w * m * k, "a"), _dev_check(b, w * k * n, "b")
        c = _dev_check(out, w * m * n, "out") if out is not None else _empty_like_kind(a, w * m * n)
        nfo = (C.c_int * 4)()
        check(getattr(L, dev_sym)(_ptr(a), _ptr(b), _ptr(c), m, k, n, arg, target, None, 0, nfo, _stream()),
              dev_sym)
        if form == "split":
            return c, {"slices": nfo[0], "rho_a": nfo[1], "rho_b": nfo[2]}
        return c, {"moduli": nfo[0], "rho_a": nfo[1], "rho_b": nfo[2], "bits": nfo[3]}
    if target != 8.0:
        raise ValueError("the host-pointer split calls use the target 8 (k 2^-104 (|A||B|)_ij units); "
                         "pass CUDA tensors for another target")
    a, b = _host(a, w * m * k, "a"), _host(b, w * k * n, "b")
    c = _host_out(out, w * m * n, "out") if out is not None else np.empty(w * m * n)
    bound = C.c_double(0.0)
    getattr(L, host_sym)(_ptr(a), _ptr(b), _ptr(c), m, k, n, arg, C.byref(bound))
    check_last(host_sym)
    return c, {"bound": bound.value}


def matmuldd_mm_split(a, b, m: int, k: int, n: int, slices: int = 0, target: float = 8.0, out=None):
    """C = A B by the digit-sliced split-INT8 form, within target k 2^-104
    (|A||B|)_ij.  Returns (C, info): the plan (slices, rho_a, rho_b) for CUDA
    tensors, the a-priori bound for host arrays."""
    return _split_call("split", False, a, b, m, k, n, slices, target, out)


def matmuldd_mm_crt(a, b, m: int, k: int, n: int, bits: int = 0, target: float = 8.0, out=None):
    """C = A B by the CRT (modular) split form; `bits` fixes the operand width W
    (0: the smallest meeting `target`).  Returns (C, info): the plan (moduli,
    rho_a, rho_b, bits) for CUDA tensors, the a-priori bound for host arrays."""
    return _split_call("crt", False, a, b, m, k, n, bits, target, out)


def cmatmuldd_mm_split(a, b, m: int, k: int, n: int, slices: int = 0, target: float = 8.0, out=None):
    """Complex (complex64x2) digit-sliced form; see matmuldd_mm_split."""
    return _split_call("split", True, a, b, m, k, n, slices, target, out)


def cmatmuldd_mm_crt(a, b, m: int, k: int, n: int, bits: int = 0, target: float = 8.0, out=None):
    """Complex (complex64x2) CRT form; see matmuldd_mm_crt."""
    return _split_call("crt", True, a, b, m, k, n, bits, target, out)


# ---- batch plans (no reference counterpart) ------------------------------------------
FORM = {"plain": 0, "split": 1, "crt": 2}


class GemmBatch:
    """A plan over many independent products of CUDA tensors, replayed as one
    CUDA-graph launch (mfcuda_batch_create_gemm / _cgemm).  problems: a list of
    (a, b, c, m, k, n); the tensors must outlive the plan, and refilling them
    between runs is how new data enters.  form: "plain", "split" or "crt";
    `slices` is the slice count (split) or the operand width (crt)."""

    def __init__(self, problems, form: str = "split", renorm_interval: int = 8, slices: int = 0,
                 target: float = 8.0, tune: bool = False, complex_: bool = False):
        from ._lib import gemm_desc

        w = 4 if complex_ else 2
        descs = (gemm_desc * max(len(problems), 1))()
        for i, (a, b, c, m, k, n) in enumerate(problems):
            if m * n:
                _dev_check(c, w * m * n, "c")
            if m * k * n:
                _dev_check(a, w * m * k, "a")
                _dev_check(b, w * k * n, "b")
            descs[i].a, descs[i].b, descs[i].c = _ptr(a) or None, _ptr(b) or None, _ptr(c) or None
            descs[i].m, descs[i].k, descs[i].n = m, k, n
        self._keep = problems
        self._plan = C.c_void_p()
        fn = "mfcuda_batch_create_cgemm" if complex_ else "mfcuda_batch_create_gemm"
        check(getattr(lib(), fn)(descs, len(problems), FORM[form], renorm_interval, slices, target, int(tune),
                                 C.byref(self._plan)), fn)

    def run(self):
        check(lib().mfcuda_batch_run(self._plan, _stream()), "mfcuda_batch_run")

    def status(self) -> int:
        """Waits for the device; MFCUDA_ERR_TIMEOUT if a bounded device wait of the last run expired."""
        return lib().mfcuda_batch_status(self._plan)

    def close(self):
        if self._plan:
            lib().mfcuda_batch_destroy(self._plan)
            self._plan = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- elementwise ---------------------------------------------------------------
def unary(op: str, x, out=None):
    """y[i] = op(x[i]) for op in exp, log, sin, cos, sqrt, exp2, log2, log10."""
    L = lib()
    code = OP[op]
    n = (x.numel() if _is_dev(x) else np.asarray(x).size) // 2
    if _is_dev(x):
        x = _dev_check(x, 2 * n, "x")
        y = _dev_check(out, 2 * n, "out") if out is not None else _empty_like_kind(x, 2 * n)
        check(L.mfcuda_unary_dd(code, _ptr(x), _ptr(y), n, _stream()), "mfcuda_unary_dd")
        return y
    x = _host(x, 2 * n, "x")
    y = _host_out(out, 2 * n, "out") if out is not None else np.empty(2 * n)
    getattr(L, f"{op}dd_array")(_ptr(x), _ptr(y), n)
    check_last(f"{op}dd_array")
    return y


def sincos(x, s=None, c=None):
    """(sin x, cos x) elementwise in one pass (sincosdd); device tensors or numpy."""
    L = lib()
    n = (x.numel() if _is_dev(x) else np.asarray(x).size) // 2
    if _is_dev(x):
        x = _dev_check(x, 2 * n, "x")
        s = _dev_check(s, 2 * n, "s") if s is not None else _empty_like_kind(x, 2 * n)
        c = _dev_check(c, 2 * n, "c") if c is not None else _empty_like_kind(x, 2 * n)
        check(L.mfcuda_sincos_dd(_ptr(x), _ptr(s), _ptr(c), n, _stream()), "mfcuda_sincos_dd")
        return s, c
    x = _host(x, 2 * n, "x")
    s = _host_out(s, 2 * n, "s") if s is not None else np.empty(2 * n)
    c = _host_out(c, 2 * n, "c") if c is not None else np.empty(2 * n)
    L.sincosdd_array(_ptr(x), _ptr(s), _ptr(c), n)
    check_last("sincosdd_array")
    return s, c


def cexpi(x, out=None):
    """cos x + i sin x as complex64x2 (cexpidd); device tensors or numpy."""
    L = lib()
    n = (x.numel() if _is_dev(x) else np.asarray(x).size) // 2
    if _is_dev(x):
        x = _dev_check(x, 2 * n, "x")
        z = _dev_check(out, 4 * n, "out") if out is not None else _empty_like_kind(x, 4 * n)
        check(L.mfcuda_cexpi_dd(_ptr(x), _ptr(z), n, _stream()), "mfcuda_cexpi_dd")
        return z
    x = _host(x, 2 * n, "x")
    z = _host_out(out, 4 * n, "out") if out is not None else np.empty(4 * n)
    L.cexpidd_array(_ptr(x), _ptr(z), n)
    check_last("cexpidd_array")
    return z


def cexp(z, out=None):
    """exp of complex64x2 elements (cexpdd); device tensors or numpy."""
    L = lib()
    n = (z.numel() if _is_dev(z) else np.asarray(z).size) // 4
    if _is_dev(z):
        z = _dev_check(z, 4 * n, "z")
        w = _dev_check(out, 4 * n, "out") if out is not None else _empty_like_kind(z, 4 * n)
        check(L.mfcuda_cexp_dd(_ptr(z), _ptr(w), n, _stream()), "mfcuda_cexp_dd")
        return w
    z = _host(z, 4 * n, "z")
    w = _host_out(out, 4 * n, "out") if out is not None else np.empty(4 * n)
    L.cexpdd_array(_ptr(z), _ptr(w), n)
    check_last("cexpdd_array")
    return w


def exp(x, out=None):
    return unary("exp", x, out)


def log(x, out=None):
    return unary("log", x, out)


def sin(x, out=None):
    return unary("sin", x, out)


def cos(x, out=None):
    return unary("cos", x, out)


def sqrt(x, out=None):
    return unary("sqrt", x, out)


# ---- reductions ----------------------------------------------------------------
def _dd_tuple(r) -> tuple:
    return (r.hi, r.lo)


def _reduce_dev(fn: str, args: list, out_doubles: int, ref):
    import torch

    L = lib()
    out = torch.empty(out_doubles, dtype=torch.float64, device=ref.device)
    check(getattr(L, fn)(*args, _ptr(out), None, 0, _stream()), fn)
    return out


def sum_dd(x):
    """Fortran sum(x) over a real64x2 array; returns (hi, lo) or a device tensor."""
    n = (x.numel() if _is_dev(x) else np.asarray(x).size) // 2
    if _is_dev(x):
        return _reduce_dev("mfcuda_sumdd", [_ptr(x), n], 2, x)
    x = _host(x, 2 * n, "x")
    r = lib().sumdd_array(_ptr(x), n)
    check_last("sumdd_array")
    return _dd_tuple(r)


def dot_product(a, b, renorm_interval: int = 8):
    n = (a.numel() if _is_dev(a) else np.asarray(a).size) // 2
    if _is_dev(a):
        return _reduce_dev("mfcuda_dotdd", [_ptr(a), _ptr(b), n, renorm_interval], 2, a)
    a, b = _host(a, 2 * n, "a"), _host(b, 2 * n, "b")
    r = lib().dotdd_array(_ptr(a), _ptr(b), n, renorm_interval)
    check_last("dotdd_array")
    return _dd_tuple(r)


def norm2(x):
    n = (x.numel() if _is_dev(x) else np.asarray(x).size) // 2
    if _is_dev(x):
        return _reduce_dev("mfcuda_norm2dd", [_ptr(x), n], 2, x)
    x = _host(x, 2 * n, "x")
    r = lib().norm2dd_array(_ptr(x), n)
    check_last("norm2dd_array")
    return _dd_tuple(r)


def csum_dd(x):
    n = (x.numel() if _is_dev(x) else np.asarray(x).size) // 4
    if _is_dev(x):
        return _reduce_dev("mfcuda_csumdd", [_ptr(x), n], 4, x)
    x = _host(x, 4 * n, "x")
    r = lib().csumdd_array(_ptr(x), n)
    check_last("csumdd_array")
    return (r.re.hi, r.re.lo, r.im.hi, r.im.lo)


def cdot_product(a, b, renorm_interval: int = 8):
    """conj(a) . b (Fortran dot_product on cmplx64x2)."""
    n = (a.numel() if _is_dev(a) else np.asarray(a).size) // 4
    if _is_dev(a):
        return _reduce_dev("mfcuda_cdotdd", [_ptr(a), _ptr(b), n, renorm_interval], 4, a)
    a, b = _host(a, 4 * n, "a"), _host(b, 4 * n, "b")
    r = lib().cdotdd_array(_ptr(a), _ptr(b), n, renorm_interval)
    check_last("cdotdd_array")
    return (r.re.hi, r.re.lo, r.im.hi, r.im.lo)


def cnorm2(x):
    n = (x.numel() if _is_dev(x) else np.asarray(x).size) // 4
    if _is_dev(x):
        return _reduce_dev("mfcuda_cnorm2dd", [_ptr(x), n], 2, x)
    x = _host(x, 4 * n, "x")
    r = lib().cnorm2dd_array(_ptr(x), n)
    check_last("cnorm2dd_array")
    return _dd_tuple(r)


def reduce_geometry(n: int) -> tuple[int, int]:
    b, t = C.c_int64(), C.c_int64()
    lib().mfcuda_reduce_geometry(n, C.byref(b), C.byref(t))
    return b.value, t.value


__all__ = [
    "matmuldd_mm", "matmuldd_mv", "matmuldd_vm", "cmatmuldd_mm",
    "unary", "exp", "log", "sin", "cos", "sqrt",
    "sum_dd", "dot_product", "norm2", "csum_dd", "cdot_product", "cnorm2",
    "reduce_geometry", "float64x2", "complex64x2",
]


# ---- BLAS-style shims (wgemm / wtrsm) ---------------------------------------------
class BlasArgumentError(ValueError):
    """An invalid wgemm / wtrsm argument: `info` is the BLAS parameter position
    (the code the reference shims hand to xerbla)."""

    def __init__(self, name: str, info: int):
        self.info = info
        super().__init__(f"{name}: parameter number {info} had an illegal value")


def _dd_scalar(v) -> np.ndarray:
    s = np.zeros(2, dtype=np.float64)
    a = np.asarray(v, dtype=np.float64).reshape(-1)
    s[: a.size] = a[:2]
    return s


def _span(ld: int, rows: int, cols: int) -> int:
    """Doubles a column-major rows x cols DD operand spans at leading dimension ld."""
    return 0 if rows <= 0 or cols <= 0 else 2 * (ld * (cols - 1) + rows)


def _need(x, doubles: int, name: str):
    if doubles == 0:
        return x
    if x is None:
        raise ValueError(f"{name}: operand missing")
    if _is_dev(x):
        import torch

        if x.dtype != torch.float64 or not x.is_contiguous() or x.numel() < doubles:
            raise ValueError(f"{name}: expected a contiguous float64 CUDA tensor of >= {doubles} doubles")
    elif not (isinstance(x, np.ndarray) and x.dtype == np.float64 and x.flags.c_contiguous and x.size >= doubles):
        raise ValueError(f"{name}: expected a contiguous float64 array of >= {doubles} doubles")
    return x


def _ch(x: str) -> bytes:
    return str(x).encode()[:1]


def wgemm(transa: str, transb: str, m: int, n: int, k: int, alpha, a, lda: int, b, ldb: int, beta,
          c, ldc: int):
    """C := alpha op(A) op(B) + beta C in place, DGEMM argument semantics
    (test/integration/blas/wgemm.f90): column-major DD operands with leading
    dimensions, op = 'N' | 'T' | 'C'; alpha / beta are one DD each ((hi, lo) or
    a float).  CUDA tensors go through mfcuda_wgemm_dd on torch's current
    stream, numpy arrays through the Fortran-callable wgemm_ (host pointers).
    Returns c."""
    L = lib()
    al, be = _dd_scalar(alpha), _dd_scalar(beta)
    info = C.c_int(0)
    scalars = (_ch(transa), _ch(transb), m, n, k)
    nota, notb = _ch(transa).upper() == b"N", _ch(transb).upper() == b"N"
    # argument check only: with no operands the call returns before any device work
    L.mfcuda_wgemm_dd(*scalars, al.ctypes.data, None, lda, None, ldb, be.ctypes.data, None, ldc,
                      C.byref(info), None)
    if info.value:
        raise BlasArgumentError("wgemm", info.value)
    if m == 0 or n == 0:
        return c  # wgemm.f90:49
    uses_ab = not (al[0] == 0.0 and al[1] == 0.0)  # alpha = 0: A and B are not read
    a = _need(a, _span(lda, m if nota else k, k if nota else m) if uses_ab else 0, "a")
    b = _need(b, _span(ldb, k if notb else n, n if notb else k) if uses_ab else 0, "b")
    c = _need(c, _span(ldc, m, n), "c")
    if _is_dev(c):
        check(L.mfcuda_wgemm_dd(*scalars, al.ctypes.data, _ptr(a), lda, _ptr(b), ldb, be.ctypes.data, _ptr(c),
                                ldc, C.byref(info), _stream()), "mfcuda_wgemm_dd")
        return c
    ints = [C.c_int(v) for v in (m, n, k, lda, ldb, ldc)]
    ta, tb = C.c_char(_ch(transa)), C.c_char(_ch(transb))
    L.wgemm_(C.byref(ta), C.byref(tb), C.byref(ints[0]), C.byref(ints[1]), C.byref(ints[2]), al.ctypes.data,
             _ptr(a), C.byref(ints[3]), _ptr(b), C.byref(ints[4]), be.ctypes.data, _ptr(c), C.byref(ints[5]), 1, 1)
    check_last("wgemm_")
    return c


def wtrsm(side: str, uplo: str, transa: str, diag: str, m: int, n: int, alpha, a, lda: int, b, ldb: int):
    """B := alpha inv(op(A)) B (side 'L') or alpha B inv(op(A)) (side 'R') in
    place, DTRSM argument semantics (test/integration/blas/wtrsm.f90): A
    triangular ('U' | 'L'), unit or non-unit diagonal ('U' | 'N').  CUDA tensors
    go through mfcuda_wtrsm_dd, numpy arrays through wtrsm_.  Returns b."""
    L = lib()
    al = _dd_scalar(alpha)
    info = C.c_int(0)
    scalars = (_ch(side), _ch(uplo), _ch(transa), _ch(diag), m, n)
    # argument check only: with no operands the call returns before any device work
    L.mfcuda_wtrsm_dd(*scalars, al.ctypes.data, None, lda, None, ldb, C.byref(info), None)
    if info.value:
        raise BlasArgumentError("wtrsm", info.value)
    if m == 0 or n == 0:
        return b
    na = m if _ch(side).upper() == b"L" else n
    a = _need(a, _span(lda, na, na) if not (al[0] == 0.0 and al[1] == 0.0) else 0, "a")
    b = _need(b, _span(ldb, m, n), "b")
    if _is_dev(b):
        check(L.mfcuda_wtrsm_dd(*scalars, al.ctypes.data, _ptr(a), lda, _ptr(b), ldb, C.byref(info), _stream()),
              "mfcuda_wtrsm_dd")
        return b
    ints = [C.c_int(v) for v in (m, n, lda, ldb)]
    ch = [C.c_char(_ch(v)) for v in (side, uplo, transa, diag)]
    L.wtrsm_(*(C.byref(x) for x in ch), C.byref(ints[0]), C.byref(ints[1]), al.ctypes.data, _ptr(a),
             C.byref(ints[2]), _ptr(b), C.byref(ints[3]), 1, 1, 1, 1)
    check_last("wtrsm_")
    return b
