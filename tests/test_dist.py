"""Multi-process logic of multifloats_b200.dist on CPU (gloo, world sizes 2 and
3): shard bounds, cost-balanced assignment, the rank-order combine of
reduction partials, and column-panel GEMMs that agree on the slice count (or,
in the CRT form, on the operand width).

Each rank's local compute is the oracle (the CPU restatement of the device
kernels), so a rank here computes what a GPU rank computes, bit for bit."""
import os
import socket

import numpy as np
import pytest

from multifloats_b200 import dist as D
from multifloats_b200 import workloads as W
from oracle import oracle as O


def test_shard_bounds_cover():
    for n in (0, 1, 7, 100, 10007):
        for world in (1, 2, 3, 8):
            bounds = [D.shard_bounds(n, r, world) for r in range(world)]
            assert bounds[0][0] == 0 and bounds[-1][1] == n
            assert all(bounds[r][1] == bounds[r + 1][0] for r in range(world - 1))
            sizes = [b - a for a, b in bounds]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        D.shard_bounds(5, 2, 2)


def test_assign_by_cost_balanced_and_deterministic():
    rng = np.random.default_rng(0)
    shapes = np.exp(rng.uniform(np.log(16), np.log(1024), (2000, 3))).astype(int)
    costs = [D.gemm_cost(*s) for s in shapes]
    for world in (2, 4, 8):
        a = D.assign_by_cost(costs, world)
        assert a == D.assign_by_cost(costs, world)
        flat = sorted(i for lst in a for i in lst)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in lst) for lst in a]
        # LPT: the most loaded rank exceeds the mean by at most the largest cost
        assert max(loads) <= sum(costs) / world + max(costs)


class OracleBackend:
    """The per-rank compute of dist.CudaBackend, restated on the CPU."""

    def partial(self, kind, x, y=None, ri=8):
        import torch

        return torch.from_numpy(O.reduce_partial(kind, x.numpy(), None if y is None else y.numpy(), ri).copy())

    def combine(self, kind, parts):
        import torch

        return torch.from_numpy(O.reduce_combine(kind, parts.numpy()).copy())

    def gemm_plain(self, a, b, m, k, n, ri):
        import torch

        return torch.from_numpy(O.matmul_mm(a.numpy(), b.numpy(), m, k, n, ri).copy())

    def gemm_split(self, a, b, m, k, n, slices, target):
        import torch

        c, info = O.split_gemm(a.numpy(), b.numpy(), m, k, n, slices=slices, target=target)
        return torch.from_numpy(c.copy()), info[0]

    def gemm_crt(self, a, b, m, k, n, bits, target):
        import torch

        c, info = O.crt_gemm(a.numpy(), b.numpy(), m, k, n, bits=bits, target=target)
        return torch.from_numpy(c.copy()), info[3]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


N_RED = 10007
M, K, NCOL = 37, 90, 29
TARGET_SPLIT = 2.0 ** 20


def _split_b(k, n, world):
    """B whose column panels differ in exponent spread: the last panel's
    columns span ~9 binades, the others one, so the ranks' own slice counts
    differ at TARGET_SPLIT."""
    parts = []
    for r in range(world):
        j0, j1 = D.column_panel(n, r, world)
        w = j1 - j0
        if r == world - 1:
            parts.append(W.dd_rowcol_scaled(k, w, 4, "row", seed=40 + r))
        else:
            parts.append(W.dd_rowcol_scaled(k, w, 0, "col", seed=40 + r))
    return np.concatenate(parts)


def _worker(rank, world, port, errq):
    try:
        import torch
        import torch.distributed as dist

        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        import datetime

        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
        be = OracleBackend()
        # ---- reductions ----
        x = W.dd_uniform(N_RED, seed=1)
        y = W.dd_uniform(N_RED, seed=2)
        cx = W.dd_uniform(2 * N_RED, seed=3)
        cy = W.dd_uniform(2 * N_RED, seed=4)
        for kind in ("sum", "dot", "norm2", "csum", "cdot", "cnorm2"):
            cplx = kind.startswith("c")
            e = 4 if cplx else 2
            xs, ys = (cx, cy) if cplx else (x, y)
            a, b = D.shard_bounds(N_RED, rank, world)
            xl = torch.from_numpy(xs[e * a: e * b].copy())
            yl = torch.from_numpy(ys[e * a: e * b].copy()) if kind in ("dot", "cdot") else None
            got = D.reduce(kind, xl, yl, 8, backend=be).numpy()
            # the same order computed in one process
            parts = []
            for r in range(world):
                ra, rb = D.shard_bounds(N_RED, r, world)
                parts.append(O.reduce_partial(kind, xs[e * ra: e * rb],
                                              ys[e * ra: e * rb] if kind in ("dot", "cdot") else None, 8))
            want = O.reduce_combine(kind, np.concatenate(parts))
            assert O.same_bits(got, want).all(), (kind, got, want)
            # and within the compensated bound of the exact value
            if kind in ("sum", "dot"):
                err, scale = O.reduce_error(kind, xs, ys if kind == "dot" else None, got)
                assert abs(err) <= 16 * 2.0 ** -104 * scale, (kind, err, scale)
        # ---- plain GEMM in column panels ----
        A = W.dd_uniform(M * K, seed=10)
        B = W.dd_uniform(K * NCOL, seed=11)
        j0, j1 = D.column_panel(NCOL, rank, world)
        bl = torch.from_numpy(B[2 * K * j0: 2 * K * j1].copy())
        c, s_used = D.matmul_columns(torch.from_numpy(A), bl, M, K, j1 - j0, "plain", 8, backend=be)
        full = D.gather_columns(c, M, NCOL).numpy()
        assert O.same_bits(full, O.matmul_mm(A, B, M, K, NCOL, 8)).all()
        # ---- split GEMM: ranks agree on the slice count of the whole problem ----
        A = W.dd_rowcol_scaled(M, K, 0, "row", seed=10)  # one binade per row
        Bs = _split_b(K, NCOL, world)
        bl = torch.from_numpy(Bs[2 * K * j0: 2 * K * j1].copy())
        own = O.split_gemm(A, Bs[2 * K * j0: 2 * K * j1], M, K, j1 - j0, target=TARGET_SPLIT)[1][0]
        c, s_used = D.matmul_columns(torch.from_numpy(A), bl, M, K, j1 - j0, "split", slices=0,
                                     target=TARGET_SPLIT, backend=be)
        want, info = O.split_gemm(A, Bs, M, K, NCOL, target=TARGET_SPLIT)
        assert s_used == info[0]
        full = D.gather_columns(c, M, NCOL).numpy()
        assert O.same_bits(full, want).all()
        # the test is only meaningful if some rank's own count differed
        flags = torch.tensor([int(own != info[0])])
        dist.all_reduce(flags)
        assert int(flags.item()) >= 1
        # ---- CRT form: ranks agree on the operand width of the whole problem ----
        own_w = O.crt_gemm(A, Bs[2 * K * j0: 2 * K * j1], M, K, j1 - j0)[1][3]
        c, w_used = D.matmul_columns(torch.from_numpy(A), bl, M, K, j1 - j0, "crt", backend=be)
        want, info = O.crt_gemm(A, Bs, M, K, NCOL)
        assert w_used == info[3]
        assert O.same_bits(D.gather_columns(c, M, NCOL).numpy(), want).all()
        flags = torch.tensor([int(own_w != info[3])])
        dist.all_reduce(flags)
        assert int(flags.item()) >= 1
        dist.barrier()
        dist.destroy_process_group()
    except BaseException as exc:  # reported to the parent
        import traceback

        errq.put((rank, traceback.format_exc()))
        raise SystemExit(1) from exc


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks(world):
    import multiprocessing as mp

    O.orc()  # build the oracle once before the ranks start
    ctx = mp.get_context("spawn")
    errq = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, errq)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
    alive = [p for p in procs if p.is_alive()]
    for p in alive:
        p.kill()
    errors = []
    while not errq.empty():
        errors.append(errq.get())
    assert not alive, "a rank did not finish"
    assert not errors, errors
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
