"""Helpers of the sharded-run tests: split a workload by detectors and run a
function on world_size ranks joined by a gloo process group on 127.0.0.1."""
import os
import socket

import numpy as np


def shard(d, rank, nranks):
    """The detectors rank r holds (round robin) with their TOD and PSDs."""
    ndet = len(d["dets"])
    mine = [i for i in range(ndet) if i % nranks == rank]
    nsamp = d["timestamps"].size
    npsd = np.asarray(d["npsd"])
    starts = np.concatenate([[0], np.cumsum(npsd)])
    nbin = np.asarray(d["psdfreqs"]).size
    psdvals = np.asarray(d["psdvals"]).reshape(-1, nbin)
    out = dict(d)
    out["dets"] = [d["dets"][i] for i in mine]
    out["detweights"] = np.asarray(d["detweights"])[mine]
    out["pixels"] = d["pixels"].reshape(ndet, nsamp)[mine].copy()
    out["pixweights"] = d["pixweights"].reshape(ndet, nsamp, -1)[mine].copy()
    out["signal"] = d["signal"].reshape(ndet, nsamp)[mine].copy()
    out["npsd"] = npsd[mine]
    sel = np.concatenate([np.arange(starts[i], starts[i + 1]) for i in mine])
    out["psdstarts"] = np.asarray(d["psdstarts"])[sel]
    out["psdvals"] = psdvals[sel].reshape(-1)
    out["mine"] = mine
    return out


def shard_time(d, rank, nranks):
    """Every detector, and the pointing periods rank r holds (contiguous
    blocks of periods), as the reference's ranks hold time slices."""
    nsamp = d["timestamps"].size
    ndet = len(d["dets"])
    per = list(np.asarray(d["periods"])) + [nsamp]
    nper = len(per) - 1
    assert nper % nranks == 0
    k = nper // nranks
    a, b = per[rank * k], per[(rank + 1) * k]
    out = dict(d)
    out["timestamps"] = d["timestamps"][a:b].copy()
    out["pixels"] = d["pixels"].reshape(ndet, nsamp)[:, a:b].copy()
    out["pixweights"] = d["pixweights"].reshape(ndet, nsamp, -1)[:, a:b].copy()
    out["signal"] = d["signal"].reshape(ndet, nsamp)[:, a:b].copy()
    out["periods"] = np.asarray(per[rank * k:(rank + 1) * k], dtype=np.int64) - a
    out["span"] = (a, b)
    return out


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _entry(rank, world, port, fn, args):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        fn(rank, world, *args)
    finally:
        dist.destroy_process_group()


def run_ranks(fn, world=2, args=()):
    """fn(rank, world, *args) on `world` spawned processes (gloo)."""
    import torch.multiprocessing as mp
    mp.spawn(_entry, args=(world, free_port(), fn, args), nprocs=world, join=True)


def gloo_allreduce(a, op):
    """In-place all-reduce of a float64 numpy array over the gloo group."""
    import torch
    import torch.distributed as dist
    t = torch.from_numpy(a)
    dist.all_reduce(t, op=dist.ReduceOp.SUM if op == 0 else dist.ReduceOp.MAX)
