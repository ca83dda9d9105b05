"""The no-allocation pixel-matrix entry point against destripe's own products.

madam_b200_pixel_matrices_noalloc computes hit counts and inverse pixel
matrices of a device-resident pointing in a fixed device scratch array,
allocating no device memory.  Two calls in a row must reproduce the
"hits" of destripe() exactly and its "cc" within CC_RTOL of each pixel
matrix's largest entry (the sums run in a different order: global atomics
into the scratch array instead of pixel-tiled shared-memory sums), and the
second call must leave the device's free memory unchanged.  This file runs
last so that it also passes after every other GPU test.
"""
import ctypes as ct

import numpy as np
import pytest

from libmadam_b200 import _lib
from libmadam_b200 import synthetic as syn

pytestmark = pytest.mark.gpu

CC_RTOL = 1e-9


@pytest.fixture(scope="module")
def torch():
    t = pytest.importorskip("torch")
    if not t.cuda.is_available():
        pytest.skip("no CUDA device")
    return t


def _entry():
    f = _lib.load().madam_b200_pixel_matrices_noalloc
    f.restype = ct.c_int
    f.argtypes = [ct.c_long, ct.c_long, ct.c_long, ct.c_long, ct.c_void_p, ct.c_void_p,
                  ct.c_void_p, ct.c_long, ct.c_double, ct.c_void_p, ct.c_void_p, ct.c_void_p,
                  ct.c_char_p, ct.c_long]
    return f


def _call(torch, nside, nnz, detw, pix, pw, pixmode, pixlim, hits, cc):
    ndet, nsamp = pix.shape
    err = ct.create_string_buffer(256)
    st = _entry()(nside, nnz, ndet, nsamp, detw.data_ptr(), pix.data_ptr(), pw.data_ptr(),
                  pixmode, pixlim, hits.data_ptr(), cc.data_ptr(), None, err, 256)
    return st, err.value.decode()


def _check_cc(cc, ref, nnz):
    a = cc.reshape(-1, nnz * nnz)
    b = ref.reshape(-1, nnz * nnz)
    scale = np.abs(b).max(axis=1)
    err = np.abs(a - b).max(axis=1)
    bad = err > CC_RTOL * np.maximum(scale, 1e-300)
    assert not bad.any(), (np.flatnonzero(bad)[:5], err[bad][:5], scale[bad][:5])


@pytest.mark.parametrize("temperature_only", [False, True])
def test_noalloc_matches_destripe_twice(torch, temperature_only):
    from libmadam_b200 import libmadam_wrapper as W
    cfg = syn.small_config(ndet=4, nsamp_obs=1 << 15, nobs=2, nside=64, seed=31,
                           temperature_only=temperature_only)
    d = syn.generate(cfg, device="cuda")
    nside, nnz = cfg.nside, d["nnz"]
    npix = 12 * nside * nside
    pix = d["pixels"].to(torch.int64)
    pw = d["pixweights"].to(torch.float64)
    detw = torch.ones(cfg.ndet, dtype=torch.float64, device="cuda")
    hits = torch.empty(npix, dtype=torch.int32, device="cuda")
    cc = torch.empty(npix * nnz * nnz, dtype=torch.float64, device="cuda")
    # unit detector weights on both sides (mode_detweight = 1)
    pars = dict(d["pars"], mode_detweight=1)
    W.destripe(None, pars, d["dets"], d["detweights"], d["timestamps"],
               d["pixels"].reshape(-1), d["pixweights"].reshape(-1), d["signal"].reshape(-1),
               d["periods"], d["npsd"], d["psdstarts"], d["psdfreqs"], d["psdvals"])
    torch.cuda.synchronize()
    ref_hits = W.get_result("hits").reshape(-1)
    ref_cc = W.get_result("cc").reshape(-1)
    assert ref_hits.sum() > 0
    for k in range(2):
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        st, msg = _call(torch, nside, nnz, detw, pix, pw, 2, 1e-6, hits, cc)
        torch.cuda.synchronize()
        free1 = torch.cuda.mem_get_info()[0]
        assert st == 0, msg
        if k == 1:
            assert free1 == free0, (free0, free1)
        np.testing.assert_array_equal(hits.cpu().numpy(), ref_hits)
        _check_cc(cc.cpu().numpy(), ref_cc, nnz)


def test_noalloc_rejects_maps_beyond_the_scratch(torch):
    pix = torch.zeros((1, 8), dtype=torch.int64, device="cuda")
    pw = torch.ones((1, 8, 3), dtype=torch.float64, device="cuda")
    detw = torch.ones(1, dtype=torch.float64, device="cuda")
    hits = torch.empty(16, dtype=torch.int32, device="cuda")
    cc = torch.empty(16 * 9, dtype=torch.float64, device="cuda")
    st, msg = _call(torch, 128, 3, detw, pix, pw, 2, 1e-6, hits, cc)
    assert st == 1
    assert "exceeds the fixed scratch of 49152 pixels" in msg
    st, msg = _call(torch, 16, 3, detw, pix.cpu(), pw, 2, 1e-6, hits, cc)
    assert st == 1 and "device memory" in msg
