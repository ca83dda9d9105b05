"""Subchunk passes (nsubchunk > 1; smadam.F90:192-437) on the GPU against the
oracle: every pass's destriped and binned maps, hits and masks, and the
full-data pass, with subsets binned inside the passes; the FITS names carry
the subchunk (add_subchunk_id, smadam.F90:1285-1314).  Tolerances as in
test_gpu_parity: hits and masks bit-exact, binned maps 1e-10, destriped maps
1e-6 relative to the largest magnitude."""
import os

import numpy as np
import pytest

import parity
import oracle_api as O
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


def _close(a, b, rtol, what=""):
    return parity.close(a, b, rtol, what)


def _both(W, d, pars):
    args = lambda x: (pars, x["dets"], x["detweights"], x["timestamps"], x["pixels"],
                      x["pixweights"], x["signal"], x["periods"], x["npsd"], x["psdstarts"],
                      x["psdfreqs"], x["psdvals"])
    do = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in d.items()}
    dp = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in d.items()}
    O.destripe(*args(do))
    W.destripe(None, *args(dp))
    np.testing.assert_array_equal(dp["pixels"], do["pixels"])
    return do, dp


@pytest.mark.parametrize("nsub,extra", [(2, {}), (3, dict(temperature_only=True)),
                                        (2, dict(isubchunk=1))])
def test_subchunk_passes_match_oracle(W, tmp_path, nsub, extra):
    tonly = extra.get("temperature_only", False)
    cfg = syn.small_config(seed=91 + nsub, temperature_only=tonly)
    d = syn.to_numpy(syn.generate(cfg, nnz=1 if tonly else None))
    t = d["timestamps"]
    pars = dict(d["pars"], nsubchunk=nsub, path_output=str(tmp_path) + "/", write_map=True,
                write_hits=True, bin_subsets=True,
                survey=["hm1 : {} - {}".format(t[0], t[len(t) // 2])], **extra)
    do, dp = _both(W, d, pars)
    first = extra.get("isubchunk", 0)
    passes = [(c + 1) % (nsub + 1) for c in range(first, nsub + 1)]
    for isub in passes:
        pre = "subchunk_%s:%d" if isub else "%s"
        names = {k: (pre % (k, isub) if isub else k) for k in ("hits", "mask", "binmap", "map")}
        np.testing.assert_array_equal(W.get_result(names["hits"]), O.result(names["hits"]))
        np.testing.assert_array_equal(W.get_result(names["mask"]), O.result(names["mask"]))
        _close(W.get_result(names["binmap"]), O.result(names["binmap"]), 1e-10)
        _close(W.get_result(names["map"]), O.result(names["map"]), 1e-6)
        sname = ("subchunk:%d/" % isub if isub else "") + "subset_hits:0"
        np.testing.assert_array_equal(W.get_result(sname), O.result(sname))
    _close(dp["signal"], do["signal"], 1e-9)
    files = os.listdir(tmp_path)
    for isub in passes:
        tag = "_sub%dof%d" % (isub, nsub) if isub else ""
        assert "madam_hmap%s.fits" % tag in files
        assert "madam_hm1_hmap%s.fits" % tag in files
    if first == 0:
        tot = sum(W.get_result("subchunk_hits:%d" % i) for i in range(1, nsub + 1))
        np.testing.assert_array_equal(tot, W.get_result("hits"))


def test_good_baseline_fraction_with_subchunks_is_refused(W):
    d = syn.to_numpy(syn.generate(syn.small_config(seed=95)))
    pars = dict(d["pars"], nsubchunk=2, good_baseline_fraction=0.5, kfilter=False)
    with pytest.raises(RuntimeError, match="nsubchunk"):
        W.destripe(None, pars, d["dets"], d["detweights"], d["timestamps"], d["pixels"],
                   d["pixweights"], d["signal"], d["periods"], d["npsd"], d["psdstarts"],
                   d["psdfreqs"], d["psdvals"])
