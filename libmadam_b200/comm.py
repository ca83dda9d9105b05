"""Communicators of runs sharded over several ranks (one process per GPU).

The reference takes an MPI communicator (`comm.py2f()`) and sums its maps
and inner products across the ranks, each of which holds its own share of
the TOD.  Here a communicator is created once per process and passed as
`comm` to libmadam_wrapper.destripe / destripe_with_cache:

    import torch.distributed as dist
    dist.init_process_group("nccl", ...)        # one rank per GPU
    comm = NcclComm()                           # NCCL over NVLink / NVSwitch
    W.destripe(comm, pars, my_dets, ...)        # this rank's detectors / spans

Every rank then holds the whole maps (hits, binned and destriped maps are
the same on all ranks) and its own baselines; FITS files are written by
rank 0.  HostComm reduces through a CPU process group (gloo) instead, which
also runs a sharded job with several ranks on one GPU.
"""
import ctypes as ct

import numpy as np

from . import _lib

HOST_ALLREDUCE = ct.CFUNCTYPE(None, ct.POINTER(ct.c_double), ct.c_long, ct.c_int)


def _L():
    L = _lib.load()
    if not getattr(L, "_comm_ready", False):
        L.madam_b200_comm_nccl_id.restype = ct.c_int
        L.madam_b200_comm_nccl_id.argtypes = [ct.c_char_p]
        L.madam_b200_comm_init_nccl.restype = ct.c_int
        L.madam_b200_comm_init_nccl.argtypes = [ct.c_int, ct.c_int, ct.c_char_p]
        L.madam_b200_comm_init_host.restype = ct.c_int
        L.madam_b200_comm_init_host.argtypes = [ct.c_int, ct.c_int, HOST_ALLREDUCE]
        L.madam_b200_comm_free.restype = ct.c_int
        L.madam_b200_comm_free.argtypes = [ct.c_int]
        L.madam_b200_comm_error.restype = ct.c_int
        L.madam_b200_comm_error.argtypes = [ct.c_char_p, ct.c_long]
        L._comm_ready = True
    return L


def _err(L):
    b = ct.create_string_buffer(512)
    L.madam_b200_comm_error(b, 512)
    return b.value.decode()


class _Comm:
    handle = 0

    def py2f(self):
        """The handle destripe() takes as its `comm` (the reference passes
        an MPI communicator's Fortran handle there)."""
        return self.handle

    def free(self):
        if self.handle > 0:
            _L().madam_b200_comm_free(self.handle)
            self.handle = 0

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class NcclComm(_Comm):
    """NCCL communicator of rank `rank` of `nranks` (defaults: the
    torch.distributed group's); the NCCL unique id travels from rank 0 over
    that group unless given."""

    def __init__(self, rank=None, nranks=None, unique_id=None):
        L = _L()
        if rank is None or nranks is None:
            import torch.distributed as dist
            rank, nranks = dist.get_rank(), dist.get_world_size()
        if unique_id is None:
            uid = ct.create_string_buffer(128)
            if rank == 0 and L.madam_b200_comm_nccl_id(uid) != 0:
                raise RuntimeError("libmadam_b200: " + _err(L))
            unique_id = uid.raw
            if nranks > 1:
                import torch.distributed as dist
                box = [unique_id]
                dist.broadcast_object_list(box, src=0)
                unique_id = box[0]
        self.rank, self.nranks = rank, nranks
        self.handle = L.madam_b200_comm_init_nccl(rank, nranks, bytes(unique_id))
        if self.handle < 0:
            raise RuntimeError("libmadam_b200: " + _err(L))


class HostComm(_Comm):
    """Reductions through a torch.distributed CPU group (gloo): the library
    copies each buffer to host memory, this object all-reduces it."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self._group = group
        self.rank, self.nranks = dist.get_rank(group), dist.get_world_size(group)

        def reduce(ptr, n, op):
            import torch
            a = np.ctypeslib.as_array(ptr, shape=(n,))
            t = torch.from_numpy(a)
            dist.all_reduce(t, op=dist.ReduceOp.SUM if op == 0 else dist.ReduceOp.MAX,
                            group=self._group)

        self._fn = HOST_ALLREDUCE(reduce)
        self.handle = _L().madam_b200_comm_init_host(self.rank, self.nranks, self._fn)
        if self.handle < 0:
            raise RuntimeError("libmadam_b200: " + _err(_L()))
