"""The DD array path on several GPUs: one process per GPU, torch.distributed for
the plumbing.

The reference library is single-process; this module adds what a multi-GPU
caller of the same path needs, with no data-path collective except where the
path has a real exchange step:

* element-wise maps and reductions: contiguous element shards
  (:func:`shard_bounds`);
* batches of independent GEMMs: a cost-balanced assignment of whole problems
  to ranks (:func:`assign_by_cost`), each rank then runs its own batch plan;
* one large GEMM: column panels (:func:`matmul_columns`): every rank holds A
  and its panel of B and computes its panel of C.  K is never split, so every
  output equals the single-device call bit for bit (for the split forms the
  ranks first agree on the slice count or the operand width, the one the
  single call would pick);
  :func:`gather_columns` assembles C when a caller wants it on every rank;
* reductions: the one real exchange.  Each rank reduces its shard to a few DD
  values (:func:`reduce` -> ``mfcuda_reduce_partial``), the values are
  all-gathered in rank order and folded left to right with DD addition on the
  device (``mfcuda_reduce_combine``).  A collective sum (NCCL's or gloo's)
  would round away the DD compensation, so only an all-gather moves data.
  The result is deterministic for a given world size and within the single
  call's error bound.

The per-rank compute goes through a backend object; the default one calls the
CUDA library (device tensors, current stream).  Tests substitute a CPU backend
to exercise the multi-process logic on ``gloo``.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

from . import _lib

KINDS = {"sum": 0, "dot": 1, "norm2": 2, "csum": 3, "cdot": 4, "cnorm2": 5}
# DD values per rank partial (sum/dot: the sum; norm2: the sum of squares;
# csum: re, im; cdot: rr, ii, ri, ir; cnorm2: the sum of squares)
PARTIAL_VALUES = {"sum": 1, "dot": 1, "norm2": 1, "csum": 2, "cdot": 4, "cnorm2": 1}
RESULT_DOUBLES = {"sum": 2, "dot": 2, "norm2": 2, "csum": 4, "cdot": 4, "cnorm2": 2}


def shard_bounds(n: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous shard [start, stop) of n elements for `rank` of `world`: the
    first n % world ranks get one element more."""
    if world < 1 or not 0 <= rank < world or n < 0:
        raise ValueError(f"bad shard request n={n} rank={rank} world={world}")
    q, r = divmod(n, world)
    start = rank * q + min(rank, r)
    return start, start + q + (1 if rank < r else 0)


def gemm_cost(m: int, k: int, n: int) -> float:
    """Work estimate of one DD GEMM (multiply-adds, at least 1)."""
    return float(max(1, m) * max(1, k) * max(1, n))


def assign_by_cost(costs: Sequence[float], world: int) -> list[list[int]]:
    """Longest-processing-time assignment of independent problems to ranks:
    problems in order of decreasing cost (ties by index) go to the least
    loaded rank (ties by rank).  Deterministic; each rank's list is returned
    in increasing problem index."""
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0.0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda j: (-float(costs[j]), j)):
        r = min(range(world), key=lambda q: (load[q], q))
        load[r] += float(costs[i])
        out[r].append(i)
    for lst in out:
        lst.sort()
    return out


# ---------------------------------------------------------------------------
# backends (per-rank compute)
# ---------------------------------------------------------------------------
class CudaBackend:
    """Per-rank compute on this process's GPU through the C ABI."""

    def _stream(self):
        import torch

        return C.c_void_p(torch.cuda.current_stream().cuda_stream)

    def partial(self, kind: str, x, y=None, ri: int = 8):
        import torch

        cplx = kind.startswith("c")
        n = x.numel() // (4 if cplx else 2)
        out = torch.empty(2 * PARTIAL_VALUES[kind], dtype=torch.float64, device=x.device)
        yp = y.data_ptr() if y is not None else None
        rc = _lib.lib().mfcuda_reduce_partial(KINDS[kind], x.data_ptr(), yp, n, ri, out.data_ptr(), None, 0,
                                              self._stream())
        _lib.check(rc, "mfcuda_reduce_partial")
        return out

    def combine(self, kind: str, parts):
        import torch

        out = torch.empty(RESULT_DOUBLES[kind], dtype=torch.float64, device=parts.device)
        count = parts.numel() // (2 * PARTIAL_VALUES[kind])
        rc = _lib.lib().mfcuda_reduce_combine(KINDS[kind], parts.data_ptr(), count, out.data_ptr(), self._stream())
        _lib.check(rc, "mfcuda_reduce_combine")
        return out

    def gemm_plain(self, a, b, m: int, k: int, n: int, ri: int):
        import torch

        c = torch.empty(2 * m * n, dtype=torch.float64, device=b.device)
        rc = _lib.lib().mfcuda_matmuldd_mm(a.data_ptr(), b.data_ptr(), c.data_ptr(), m, k, n, ri, self._stream())
        _lib.check(rc, "mfcuda_matmuldd_mm")
        return c

    def gemm_split(self, a, b, m: int, k: int, n: int, slices: int, target: float):
        """Returns (C, slices used)."""
        import torch

        c = torch.empty(2 * m * n, dtype=torch.float64, device=b.device)
        info = (C.c_int * 3)()
        rc = _lib.lib().mfcuda_matmuldd_mm_split(a.data_ptr(), b.data_ptr(), c.data_ptr(), m, k, n, slices,
                                                 target, None, 0, info, self._stream())
        _lib.check(rc, "mfcuda_matmuldd_mm_split")
        return c, int(info[0])

    def gemm_crt(self, a, b, m: int, k: int, n: int, bits: int, target: float):
        """CRT form; returns (C, operand width W used)."""
        import torch

        c = torch.empty(2 * m * n, dtype=torch.float64, device=b.device)
        info = (C.c_int * 4)()
        rc = _lib.lib().mfcuda_matmuldd_mm_crt(a.data_ptr(), b.data_ptr(), c.data_ptr(), m, k, n, bits, target,
                                               None, 0, info, self._stream())
        _lib.check(rc, "mfcuda_matmuldd_mm_crt")
        return c, int(info[3])


_default_backend = None


def _backend(b):
    global _default_backend
    if b is not None:
        return b
    if _default_backend is None:
        _default_backend = CudaBackend()
    return _default_backend


def _group_info(group):
    import torch.distributed as dist

    return dist.get_rank(group), dist.get_world_size(group)


def _all_gather_flat(t, group):
    """Rank-ordered concatenation of equally sized 1-D tensors from all ranks."""
    import torch
    import torch.distributed as dist

    _, world = _group_info(group)
    out = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(out, t, group=group)
    return torch.cat(out)


# ---------------------------------------------------------------------------
# reductions
# ---------------------------------------------------------------------------
def reduce(kind: str, x_local, y_local=None, ri: int = 8, group=None, backend=None):
    """Fortran sum / dot_product / norm2 (kind in KINDS) of the array whose
    contiguous shard this rank holds (x_local, y_local: DD or complex DD
    interleaved, shards as :func:`shard_bounds` gives them).  Every rank
    receives the result (2 doubles, or 4 for csum / cdot).  A rank whose
    shard is empty contributes the identity partial."""
    if kind not in KINDS:
        raise ValueError(f"unknown reduction {kind!r}")
    be = _backend(backend)
    part = be.partial(kind, x_local, y_local, ri)
    parts = _all_gather_flat(part, group)
    return be.combine(kind, parts)


def sum_dd(x_local, group=None, backend=None):
    return reduce("sum", x_local, group=group, backend=backend)


def dot_product(a_local, b_local, renorm_interval: int = 8, group=None, backend=None):
    return reduce("dot", a_local, b_local, renorm_interval, group, backend)


def norm2(x_local, group=None, backend=None):
    return reduce("norm2", x_local, group=group, backend=backend)


def csum_dd(x_local, group=None, backend=None):
    return reduce("csum", x_local, group=group, backend=backend)


def cdot_product(a_local, b_local, renorm_interval: int = 8, group=None, backend=None):
    return reduce("cdot", a_local, b_local, renorm_interval, group, backend)


def cnorm2(x_local, group=None, backend=None):
    return reduce("cnorm2", x_local, group=group, backend=backend)


# ---------------------------------------------------------------------------
# one GEMM in column panels
# ---------------------------------------------------------------------------
def column_panel(n: int, rank: int, world: int) -> tuple[int, int]:
    """Columns [j0, j1) of C (and B) owned by `rank`."""
    return shard_bounds(n, rank, world)


def matmul_columns(a, b_local, m: int, k: int, n_local: int, form: str = "plain", renorm_interval: int = 8,
                   slices: int = 0, target: float = 8.0, group=None, backend=None):
    """This rank's column panel of C = A B (column-major DD): a is all of A
    (m x k), b_local this rank's k x n_local panel of B.  Each output equals
    the single-device call bit for bit.  form "split": with slices = 0 every
    rank first runs with its own automatic slice count and the ranks agree on
    the largest one (the count the single call derives from the exponent
    spreads of all of B); a rank that used fewer recomputes with that count
    (`target` as in mfcuda_matmuldd_mm_split).  form "crt" (the CRT split
    form): the same agreement on the operand width W (`slices` is then the
    width, 0 = from the target; the single call's W grows with the spreads, so
    it is the ranks' largest).  Returns (C panel, slices or W used, 0 for the
    plain form)."""
    import torch
    import torch.distributed as dist

    be = _backend(backend)
    if form == "plain":
        if n_local == 0:
            return b_local.new_empty(0), 0
        return be.gemm_plain(a, b_local, m, k, n_local, renorm_interval), 0
    if form not in ("split", "crt"):
        raise ValueError(f"unknown form {form!r}")
    run = be.gemm_split if form == "split" else be.gemm_crt
    if n_local > 0:
        c, s_used = run(a, b_local, m, k, n_local, slices, target)
    else:
        c, s_used = b_local.new_empty(0), 0
    if slices == 0:
        s = torch.tensor([s_used], dtype=torch.int64, device=b_local.device)
        dist.all_reduce(s, op=dist.ReduceOp.MAX, group=group)
        s_all = int(s.item())
        if n_local > 0 and s_used != s_all:
            c, s_used = run(a, b_local, m, k, n_local, s_all, target)
    return c, s_used


def gather_columns(c_local, m: int, n: int, group=None):
    """Assembles the column panels of an m x n DD matrix (column-major, so a
    panel is a contiguous block) on every rank, in rank order."""
    import torch

    rank, world = _group_info(group)
    width = max(column_panel(n, r, world)[1] - column_panel(n, r, world)[0] for r in range(world))
    buf = torch.zeros(2 * m * width, dtype=torch.float64, device=c_local.device)
    buf[: c_local.numel()] = c_local
    full = _all_gather_flat(buf, group).reshape(world, -1)
    pieces = []
    for r in range(world):
        j0, j1 = column_panel(n, r, world)
        pieces.append(full[r, : 2 * m * (j1 - j0)])
    return torch.cat(pieces)
