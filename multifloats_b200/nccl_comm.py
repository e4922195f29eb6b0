"""An NCCL communicator for the library's sharded entry points
(mfcuda_matmuldd_mm_nccl, mfcuda_reduce_nccl), made through ctypes from the
NCCL library the process already loaded (torch's, when torch is imported), so
that the communicator and the library's calls use one NCCL.

    comm = NcclComm.single()                       # one rank, the current device
    comm = NcclComm.from_process_group(rank, world)  # one per rank; needs an
                                                   # initialised torch.distributed
                                                   # group to pass the unique id
    lib.mfcuda_matmuldd_mm_nccl(..., comm.handle, stream)
    comm.close()
"""
from __future__ import annotations

import ctypes as C


class _UniqueId(C.Structure):
    _fields_ = [("internal", C.c_char * 128)]


def _nccl():
    lib = C.CDLL("libnccl.so.2")
    lib.ncclGetUniqueId.argtypes = [C.POINTER(_UniqueId)]
    lib.ncclCommInitRank.argtypes = [C.POINTER(C.c_void_p), C.c_int, _UniqueId, C.c_int]
    lib.ncclCommInitAll.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.POINTER(C.c_int)]
    lib.ncclCommDestroy.argtypes = [C.c_void_p]
    lib.ncclGetErrorString.restype = C.c_char_p
    return lib


class NcclComm:
    def __init__(self, handle: C.c_void_p, lib):
        self.handle = handle
        self._lib = lib

    @classmethod
    def single(cls, device: int = 0) -> "NcclComm":
        lib = _nccl()
        comm = C.c_void_p()
        dev = (C.c_int * 1)(device)
        rc = lib.ncclCommInitAll(C.byref(comm), 1, dev)
        if rc != 0:
            raise RuntimeError(f"ncclCommInitAll: {lib.ncclGetErrorString(rc).decode()}")
        return cls(comm, lib)

    @classmethod
    def from_process_group(cls, rank: int, world: int) -> "NcclComm":
        """One communicator over the ranks of the default torch.distributed
        group (rank 0's unique id is broadcast through it); the current CUDA
        device is this rank's."""
        import torch
        import torch.distributed as dist

        lib = _nccl()
        uid = _UniqueId()
        if rank == 0:
            rc = lib.ncclGetUniqueId(C.byref(uid))
            if rc != 0:
                raise RuntimeError(f"ncclGetUniqueId: {lib.ncclGetErrorString(rc).decode()}")
        raw = torch.frombuffer(bytearray(C.string_at(C.addressof(uid), 128)), dtype=torch.uint8)
        t = raw.to("cuda") if dist.get_backend() == "nccl" else raw.clone()
        dist.broadcast(t, src=0)
        C.memmove(C.addressof(uid), t.cpu().numpy().tobytes(), 128)
        comm = C.c_void_p()
        rc = lib.ncclCommInitRank(C.byref(comm), world, uid, rank)
        if rc != 0:
            raise RuntimeError(f"ncclCommInitRank: {lib.ncclGetErrorString(rc).decode()}")
        return cls(comm, lib)

    def close(self) -> None:
        if self.handle:
            self._lib.ncclCommDestroy(self.handle)
            self.handle = None
