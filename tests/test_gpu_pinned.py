"""destripe() from page-locked host buffers: the signal is read over the bus
by a kernel on a second stream while the pointing setup runs; the products
equal those of the same call from pageable buffers (to the rounding of the
setup's float64 atomic sums), the cleaned signal is written back, and a
call that fails after the upload started leaves the engine usable."""
import numpy as np
import pytest

import parity
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


def _pinned(a):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    return t, t.numpy()


def _call(W, d, pars, ts, pix, w, sig):
    W.destripe(None, pars, d["dets"], d["detweights"], ts, pix, w, sig, d["periods"], d["npsd"],
               d["psdstarts"], d["psdfreqs"], d["psdvals"])


def test_pinned_buffers_match_pageable(W):
    d = syn.to_numpy(syn.generate(syn.small_config(seed=181, nsamp_obs=1 << 15)))
    pars = dict(d["pars"], write_tod=True)
    sig_a = d["signal"].copy()
    _call(W, d, pars, d["timestamps"].copy(), d["pixels"].copy(), d["pixweights"].copy(), sig_a)
    ref = {k: W.get_result(k) for k in ("map", "binmap", "aa", "hits")}
    keep = [_pinned(d[k]) for k in ("timestamps", "pixels", "pixweights", "signal")]
    ts, pix, w, sig = (k[1] for k in keep)
    _call(W, d, pars, ts, pix, w, sig)
    np.testing.assert_array_equal(W.get_result("hits"), ref["hits"])
    for k in ("map", "binmap", "aa"):
        _close(W.get_result(k), ref[k], 1e-8)
    # the cleaned TOD came back into the page-locked buffer
    _close(sig, sig_a, 1e-8)
    np.testing.assert_array_equal(pix, d["pixels"])


def test_failed_call_after_upload_leaves_engine_usable(W):
    d = syn.to_numpy(syn.generate(syn.small_config(seed=182)))
    keep = [_pinned(d[k]) for k in ("timestamps", "pixels", "pixweights", "signal")]
    ts, pix, w, sig = (k[1] for k in keep)
    with pytest.raises(RuntimeError, match="Unknown parameter"):
        _call(W, d, dict(d["pars"], no_such_key=1), ts, pix, w, sig)
    with pytest.raises(RuntimeError, match="nside_cross > nside_map"):
        _call(W, d, dict(d["pars"], nside_cross=2 * d["pars"]["nside_map"]), ts, pix, w, sig)
    _call(W, d, d["pars"], ts, pix, w, sig)
    assert W.scalars()["noiter"] > 0
