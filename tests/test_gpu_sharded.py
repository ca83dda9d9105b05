"""Sharded runs on the GPU: an NCCL communicator of one rank gives the
plain single-rank products, and two ranks that reduce through a CPU process
group (HostComm over gloo; two processes sharing the one GPU, synchronised
on the host, never by waiting kernels) give the products of one rank on all
the data - sharded by detector, and by time with subsets and leakage
matrices.  Tolerances: hits and masks bit-exact, maps 1e-9 relative to the
largest magnitude (the ranks' partial sums add in another order)."""
import numpy as np
import pytest

import parity
import shard_util as SU
from libmadam_b200 import synthetic as syn

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def W():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from libmadam_b200 import libmadam_wrapper
    assert libmadam_wrapper.available
    return libmadam_wrapper


def _args(pars, x):
    return (pars, x["dets"], x["detweights"], x["timestamps"], x["pixels"], x["pixweights"],
            x["signal"], x["periods"], x["npsd"], x["psdstarts"], x["psdfreqs"], x["psdvals"])


def _close(a, b, rtol, what=""):
    return parity.close(a, b, rtol, what)


def test_nccl_single_rank_matches_plain(W):
    from libmadam_b200.comm import NcclComm
    d = syn.to_numpy(syn.generate(syn.small_config(seed=111)))
    full = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in d.items()}
    W.destripe(None, *_args(d["pars"], full))
    ref = {k: W.get_result(k) for k in ("map", "binmap", "hits", "aa")}
    comm = NcclComm(0, 1)
    again = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in d.items()}
    W.destripe(comm, *_args(d["pars"], again))
    np.testing.assert_array_equal(W.get_result("hits"), ref["hits"])
    for k in ("map", "binmap", "aa"):
        _close(W.get_result(k), ref[k], 1e-10)
    comm.free()


def _rank(rank, world, by_time):
    import torch
    from libmadam_b200 import libmadam_wrapper as W
    from libmadam_b200.comm import HostComm
    torch.cuda.set_device(0)
    d = syn.to_numpy(syn.generate(syn.small_config(seed=112)))
    pars = dict(d["pars"])
    if by_time:
        t = d["timestamps"]
        pars.update(bin_subsets=True, write_leakmatrix=True,
                    survey=["hm1 : {} - {}".format(t[0], t[len(t) // 2])],
                    detset=["AB : det000, det001"])
    full = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in d.items()}
    W.destripe(None, *_args(pars, full))
    ref = {k: W.get_result(k) for k in ("map", "binmap", "hits", "mask")}
    if by_time:
        ref_sub = W.get_result("subset_binmap:0")
        ref_leak = W.get_result("leakmatrix:1")
    ref_it = W.scalars()["noiter"]
    mine = SU.shard_time(d, rank, world) if by_time else SU.shard(d, rank, world)
    comm = HostComm()
    W.destripe(comm, *_args(pars, mine))
    np.testing.assert_array_equal(W.get_result("hits"), ref["hits"])
    np.testing.assert_array_equal(W.get_result("mask"), ref["mask"])
    _close(W.get_result("map"), ref["map"], 1e-9)
    _close(W.get_result("binmap"), ref["binmap"], 1e-9)
    assert W.scalars()["noiter"] == ref_it
    if by_time:
        _close(W.get_result("subset_binmap:0"), ref_sub, 1e-9)
        np.testing.assert_allclose(W.get_result("leakmatrix:1"), ref_leak, rtol=0, atol=1e-8)
    comm.free()


def test_two_ranks_by_detector_on_one_gpu(W):
    SU.run_ranks(_rank, 2, (False,))


def test_two_ranks_by_time_with_subsets_on_one_gpu(W):
    SU.run_ranks(_rank, 2, (True,))


def _covmat_rank(rank, world, root):
    import torch
    from libmadam_b200 import libmadam_wrapper as W
    from libmadam_b200.comm import HostComm
    from test_oracle_covmat import _data, read_covmat
    torch.cuda.set_device(0)
    d = _data(174)
    N = 12 * d["pars"]["nside_map"] ** 2 * 3
    full = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in d.items()}
    W.destripe(None, *_args(dict(d["pars"], file_covmat="{}_full{}".format(root, rank)), full))
    mine = SU.shard_time(d, rank, world)
    comm = HostComm()
    W.destripe(comm, *_args(dict(d["pars"], file_covmat=root + "_shard"), mine))
    if rank == 0:
        for det in d["dets"]:
            a = read_covmat(root + "_shard", det, N)
            b = read_covmat("{}_full{}".format(root, rank), det, N)
            _close(a, b, 1e-11)


def test_two_host_ranks_covmat(W, tmp_path):
    # the ranks' covariance matrices are summed on the device arrays and
    # rank 0 writes the files
    SU.run_ranks(_covmat_rank, 2, (str(tmp_path / "ncm"),))
