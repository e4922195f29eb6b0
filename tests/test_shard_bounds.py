"""The library's shard arithmetic (mfcuda_shard_bounds, used by the NCCL
entry points to find each rank's column panel) agrees with the Python
sharding helper for every rank of several worlds, on the CPU."""
import ctypes as C

from multifloats_b200 import _lib, dist


def test_bounds_match_python_helper():
    L = _lib.lib()
    a, b = C.c_int64(), C.c_int64()
    for n in (0, 1, 7, 8, 100, 4096, 8191):
        for world in (1, 2, 3, 4, 7, 8):
            prev = 0
            for rank in range(world):
                L.mfcuda_shard_bounds(n, rank, world, C.byref(a), C.byref(b))
                assert (a.value, b.value) == dist.shard_bounds(n, rank, world)
                assert a.value == prev
                prev = b.value
            assert prev == n
    L.mfcuda_shard_bounds(5, 3, 2, C.byref(a), C.byref(b))
    assert (a.value, b.value) == (0, 0)
