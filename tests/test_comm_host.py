"""Library communicators on gloo ranks without a GPU (world size 2): ranks,
handles out of the range of MPI Fortran handles, freeing; and the
spectrum-file check that a lone rank makes before any device work is left
to the filter build on a sharded run, where every rank reports the file's
error after the same collective steps (a rank failing alone before them
would leave the others waiting)."""
import numpy as np
import pytest

import shard_util as SU


def _call(W, comm, pars):
    W.destripe(comm, pars, ["a"], np.ones(1), np.zeros(4), np.zeros(4, np.int32),
               np.ones(4, np.float32), np.zeros(4), np.array([0]), np.ones(1, np.int64),
               np.zeros(1), np.array([1.0, 2.0]), np.ones(2))


def _rank(rank, world, path):
    import torch
    import torch.distributed as dist
    from libmadam_b200 import comm as C
    from libmadam_b200 import libmadam_wrapper as W
    c = C.HostComm()
    assert (c.rank, c.nranks) == (rank, world)
    assert c.handle >= 0x2D420001
    ranks = [None] * world
    dist.all_gather_object(ranks, c.rank)
    assert ranks == list(range(world))
    bad = {"kfilter": True, "file_spectrum": path}
    with pytest.raises(RuntimeError) as e:
        _call(W, c, bad)
    msg = str(e.value)
    # a sharded rank gets past the file to the device (none here)
    assert "not in" not in msg and "CUDA" in msg, msg
    c.free()
    assert c.handle == 0
    # a lone rank (no communicator) fails on the file itself
    with pytest.raises(RuntimeError, match="ERROR: a not in"):
        _call(W, None, bad)
    dist.barrier()
    del torch


def test_host_comm_on_two_ranks(tmp_path):
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present: the device path runs in the GPU tests")
    path = tmp_path / "spec.txt"
    path.write_text("3 1\nb\n1e-3\n0.01 1e-4\n0.1 1e-5\n1.0 1e-6\n")
    SU.run_ranks(_rank, 2, (str(path),))
