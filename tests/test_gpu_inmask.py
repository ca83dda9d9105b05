"""The input mask (file_inmask) on the GPU against the oracle: FITS mask
tables at nside_cross, at a finer resolution (downgraded) and at a coarser
one (upgraded), in float32, int32 and float64 columns.  Hits and masks
bit-exact, maps and baselines within 1e-6 of their largest magnitude."""
import numpy as np
import pytest

import parity
import oracle_api as O
from fits_reader import write_mask
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


@pytest.mark.parametrize("res,code", [(16, "E"), (32, "J"), (8, "D")])
def test_inmask_matches_oracle(W, tmp_path, res, code):
    d = syn.to_numpy(syn.generate(syn.small_config(seed=131, nside=32)))
    pars = dict(d["pars"], nside_cross=16, nside_submap=4)
    rng = np.random.default_rng(res)
    f = str(tmp_path / "mask.fits")
    m = (rng.random(12 * res ** 2) > 0.15).astype(float)
    write_mask(f, m, res, code=code)
    # the mask at nside_cross 16: downgraded (any dropped sub-pixel drops the
    # pixel) or upgraded (each pixel repeated over its sub-pixels)
    keep = (m.reshape(-1, (res // 16) ** 2).min(axis=1) if res >= 16
            else np.repeat(m, (16 // res) ** 2))
    pars["file_inmask"] = f
    args = lambda x: (pars, x["dets"], x["detweights"], x["timestamps"], x["pixels"],
                      x["pixweights"], x["signal"], x["periods"], x["npsd"], x["psdstarts"],
                      x["psdfreqs"], x["psdvals"])
    do = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in d.items()}
    dp = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in d.items()}
    O.destripe(*args(do))
    W.destripe(None, *args(dp))
    np.testing.assert_array_equal(W.get_result("hits"), O.result("hits"))
    np.testing.assert_array_equal(W.get_result("mask"), O.result("mask"))
    cp = W.get_result("cca").reshape(-1, 9)
    co = O.result("cca").reshape(-1, 9)
    # the masked pixels' matrices are zero; the others agree to rounding (the
    # setup's float64 atomic sums leave ~1e-26 off-diagonals on either side)
    assert np.all(cp[keep == 0] == 0) and np.all(co[keep == 0] == 0)
    _close(cp, co, 1e-9)
    for c in range(3):
        _close(W.get_result("map").reshape(-1, 3)[:, c], O.result("map").reshape(-1, 3)[:, c],
               1e-6)
    _close(W.get_result("aa"), O.result("aa"), 1e-6)
    assert W.scalars()["noiter"] == O.scalars()["noiter"]


def test_ring_ordered_mask_is_refused(W, tmp_path):
    d = syn.to_numpy(syn.generate(syn.small_config(seed=132)))
    f = str(tmp_path / "ring.fits")
    write_mask(f, np.ones(12 * 16 ** 2), 16, ordering="RING")
    with pytest.raises(RuntimeError, match="NESTED"):
        W.destripe(None, dict(d["pars"], file_inmask=f), d["dets"], d["detweights"],
                   d["timestamps"], d["pixels"], d["pixweights"], d["signal"], d["periods"],
                   d["npsd"], d["psdstarts"], d["psdfreqs"], d["psdvals"])
