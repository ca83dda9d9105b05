"""Subset maps and leakage matrices on the GPU against the oracle
(run_subsets, smadam.F90:954-1257; leakmatrix, smadam_routines.f90:38-105).

Tolerances: hits and masks bit-exact; binned subset maps and inverted pixel
matrices within 1e-8 per element (parity.close: relative to each value, or to
1e-3 of the largest magnitude below that; both sides bin with float64 sums
in different orders, and a subset's pixel matrices, built from fewer
detectors and samples, are less well conditioned than the full data's, so
the 3x3 solves amplify those differences to a few 1e-12 of the largest
magnitude in entries near zero); leakage matrices within 1e-8 absolute
(products of inverted matrices, entries of order one)."""
import os

import numpy as np
import pytest

import parity
import oracle_api as O
from libmadam_b200 import synthetic as syn

pytestmark = pytest.mark.gpu

BIN_RTOL = 1e-8
LEAK_ATOL = 1e-8


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


def _pars(d, **kw):
    t = d["timestamps"]
    n = len(t)
    p = dict(d["pars"], bin_subsets=True, write_leakmatrix=True,
             survey=["hm1 : {} - {}".format(t[0], t[n // 2]),
                     "odd : {} - {}, {} - {}".format(t[n // 4], t[n // 2], t[3 * n // 4], t[-1])],
             detset=["AB : det000, det001", "full : all"],
             detset_nopol=["CD : det002, det003"])
    p.update(kw)
    return p


def _both(W, d, pars):
    args = lambda x: (pars, x["dets"], x["detweights"], x["timestamps"], x["pixels"],
                      x["pixweights"], x["signal"], x["periods"], x["npsd"], x["psdstarts"],
                      x["psdfreqs"], x["psdvals"])
    do = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in d.items()}
    dp = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in d.items()}
    O.destripe(*args(do))
    W.destripe(None, *args(dp))
    return do, dp


def _compare_subsets(W, ndet):
    tab_o = O.result("subsets").reshape(-1, 4)
    tab_p = W.get_result("subsets").reshape(-1, 4)
    np.testing.assert_array_equal(tab_p, tab_o)
    assert len(tab_o) > 0
    for k, (ps, _, _, nm) in enumerate(tab_o):
        nm = int(nm)
        _close(W.get_result("subset_binmap:%d" % k), O.result("subset_binmap:%d" % k), BIN_RTOL)
        if ps != 1:
            continue
        np.testing.assert_array_equal(W.get_result("subset_hits:%d" % k),
                                      O.result("subset_hits:%d" % k))
        np.testing.assert_array_equal(W.get_result("subset_mask:%d" % k),
                                      O.result("subset_mask:%d" % k))
        _close(W.get_result("subset_cc:%d" % k), O.result("subset_cc:%d" % k), BIN_RTOL)
        for det in range(ndet):
            name = "subset_leak:%d:%d" % (k, det)
            try:
                ref = O.result(name)
            except KeyError:
                with pytest.raises(KeyError):
                    W.get_result(name)
                continue
            np.testing.assert_allclose(W.get_result(name), ref, rtol=0, atol=LEAK_ATOL)
    return tab_o


def test_subsets_iqu_match_oracle(W, tmp_path):
    d = syn.to_numpy(syn.generate(syn.small_config(seed=71)))
    pars = _pars(d, path_output=str(tmp_path) + "/", file_root="sub", write_map=True,
                 write_hits=True, write_mask=True, write_matrix=True, write_wcov=True)
    do, dp = _both(W, d, pars)
    tab = _compare_subsets(W, 4)
    # 2 surveys x (full, AB, CD) + the 2 detsets alone
    assert len(tab) == 8
    assert set(tab[:, 3].tolist()) == {1.0, 3.0}
    for det in range(4):
        np.testing.assert_allclose(W.get_result("leakmatrix:%d" % det),
                                   O.result("leakmatrix:%d" % det), rtol=0, atol=LEAK_ATOL)
    # the full-data products and the cleaned TOD are those of the oracle
    _close(W.get_result("map"), O.result("map"), 1e-6)
    np.testing.assert_array_equal(W.get_result("hits"), O.result("hits"))
    _close(dp["signal"], do["signal"], 1e-9)
    files = sorted(os.listdir(tmp_path))
    assert "sub_full_map.fits" in files            # the "all" set names the full data
    assert "sub_AB_hm1_map.fits" in files and "sub_CD_odd_hmap.fits" in files
    assert "sub_full_leakmatrix_det000.fits" in files
    assert "sub_AB_hm1_leakmatrix.fits_det001.fits" in files
    assert not any(f.startswith("sub_AB_hm1_leakmatrix.fits_det002") for f in files)


def test_subsets_two_passes_and_monopole(W, tmp_path):
    d = syn.to_numpy(syn.generate(syn.small_config(seed=72)))
    pars = _pars(d, path_output=str(tmp_path) + "/", write_map=True, write_binmap=True,
                 rm_monopole=True, write_leakmatrix=False)
    _both(W, d, pars)
    tab = _compare_subsets(W, 4)
    assert set(tab[:, 0].tolist()) == {1.0, 2.0}
    files = os.listdir(tmp_path)
    assert any(f.endswith("_AB_hm1_bmap.fits") for f in files)
    assert any(f.endswith("_AB_hm1_map.fits") for f in files)


def test_subsets_temperature_only(W):
    cfg = syn.small_config(seed=73, temperature_only=True)
    d = syn.to_numpy(syn.generate(cfg, nnz=1))
    _both(W, d, _pars(d))
    tab = _compare_subsets(W, 4)
    assert set(tab[:, 3].tolist()) == {1.0}


def test_subsets_after_cached_call(W):
    d = syn.to_numpy(syn.generate(syn.small_config(seed=74)))
    pars = _pars(d, mcmode=True, write_leakmatrix=False)
    W.clear_caches()
    O.clear_caches()
    _both(W, d, pars)
    sig = d["signal"] * 0.5
    O.destripe_with_cache(d["timestamps"], d["pixels"].copy(), d["pixweights"], sig.copy(), 4)
    W.destripe_with_cache(None, d["timestamps"], d["pixels"].copy(), d["pixweights"], sig.copy(),
                          b"")
    _compare_subsets(W, 4)
    W.clear_caches()
    O.clear_caches()
