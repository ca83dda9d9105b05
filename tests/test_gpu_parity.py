"""Parity of the CUDA destriper with the CPU oracle (needs a B200).

Tolerances (FP64 path): hit counts and masks bit-exact; binned maps within
1e-10 and destriped maps / baselines within 1e-6 per pixel (per baseline) in
the sense of parity.close: relative to each value, or to 1e-3 of the
component's largest magnitude for values below that; PCG iteration counts
equal.
"""
import numpy as np
import pytest

import parity
import kat
import oracle_api as O
from libmadam_b200 import synthetic as syn

pytestmark = pytest.mark.gpu

MAP_RTOL = 1e-6
BIN_RTOL = 1e-10


@pytest.fixture(scope="module")
def W():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from libmadam_b200 import libmadam_wrapper
    assert libmadam_wrapper.available
    return libmadam_wrapper


def _copy(d):
    return {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in d.items()}


def run_both(W, d, pars=None, check_pixels=True):
    pars = dict(d["pars"], **(pars or {}))
    do, dp = _copy(d), _copy(d)
    args = lambda x: (pars, x["dets"], x["detweights"], x["timestamps"], x["pixels"],
                      x["pixweights"], x["signal"], x["periods"], x["npsd"], x["psdstarts"],
                      x["psdfreqs"], x["psdvals"])
    O.destripe(*args(do))
    ro = {k: O.result(k) for k in ("map", "binmap", "hits", "mask", "aa", "yba", "nna",
                                   "rr_history")}
    ro["scalars"] = O.scalars()
    W.destripe(None, *args(dp))
    rp = {k: W.get_result(k) for k in ("map", "binmap", "hits", "mask", "aa", "yba", "nna",
                                       "rr_history")}
    rp["scalars"] = W.scalars()
    if check_pixels:
        np.testing.assert_array_equal(dp["pixels"], do["pixels"])
    np.testing.assert_array_equal(dp["signal"], do["signal"]) if not pars.get("write_tod") else \
        _close(dp["signal"], do["signal"], 1e-9)
    return ro, rp, do, dp


def _close(a, b, rtol, what=""):
    return parity.close(a, b, rtol, what)


def compare(ro, rp, nmap, iters_exact=True):
    np.testing.assert_array_equal(rp["hits"], ro["hits"])
    np.testing.assert_array_equal(rp["mask"], ro["mask"])
    bo = ro["binmap"].reshape(-1, nmap)
    bp = rp["binmap"].reshape(-1, nmap)
    mo = ro["map"].reshape(-1, nmap)
    mp = rp["map"].reshape(-1, nmap)
    for c in range(nmap):
        _close(bp[:, c], bo[:, c], BIN_RTOL, "binmap[%d]" % c)
        _close(mp[:, c], mo[:, c], MAP_RTOL, "map[%d]" % c)
    _close(rp["nna"], ro["nna"], 1e-14, "nna")
    _close(rp["yba"], ro["yba"], 1e-9, "yba")
    _close(rp["aa"], ro["aa"], MAP_RTOL, "aa")
    if iters_exact:
        assert rp["scalars"]["noiter"] == ro["scalars"]["noiter"]
    n = min(len(ro["rr_history"]), len(rp["rr_history"]), 5)
    np.testing.assert_allclose(rp["rr_history"][:n], ro["rr_history"][:n], rtol=1e-5)


def test_reference_kat_hits_and_binned_map(W):
    from product_api import ProductBackend
    kat.run_libmadam_kat(ProductBackend(), check_files=True)


def test_reference_kat_mc_sequence(W):
    from product_api import ProductBackend
    from test_oracle_kat import OracleBackend
    mp = kat.run_mc_kat(ProductBackend(), check_files=True)
    mo = kat.run_mc_kat(OracleBackend())
    for a, b in zip(mp, mo):
        _close(a, b, MAP_RTOL)


@pytest.mark.parametrize("seed", [7, 8])
def test_ring_scan_iqu(W, seed):
    d = syn.to_numpy(syn.generate(syn.small_config(seed=seed)))
    ro, rp, _, _ = run_both(W, d)
    compare(ro, rp, 3)
    assert rp["scalars"]["noiter"] > 3


def test_ring_scan_temperature_only(W):
    cfg = syn.small_config(seed=11, temperature_only=True)
    d = syn.to_numpy(syn.generate(cfg, nnz=1))
    ro, rp, _, _ = run_both(W, d)
    compare(ro, rp, 1)


def test_flagged_samples_and_pixel_writeback(W):
    d = syn.to_numpy(syn.generate(syn.small_config(seed=12)))
    rng = np.random.default_rng(0)
    n = d["pixels"].size
    bad = rng.choice(n, n // 50, replace=False)
    d["pixweights"].reshape(-1, 3)[bad] = 0.0      # zero weight -> flagged
    d["pixels"].reshape(-1)[bad[:10]] = -1          # explicitly flagged
    ro, rp, do, dp = run_both(W, d)
    compare(ro, rp, 3)
    flagged = dp["pixels"].reshape(-1)[bad]
    assert np.all(flagged == 12 * d["pars"]["nside_map"] ** 2)


def test_sparse_period_is_flagged(W):
    d = syn.to_numpy(syn.generate(syn.small_config(seed=13)))
    # leave 5 good samples in the second period of detector 1
    per = d["periods"]
    w = d["pixweights"].reshape(4, -1, 3)
    w[1, per[1]:, :] = 0
    w[1, per[1]:per[1] + 5, :] = 1
    ro, rp, do, dp = run_both(W, d)
    compare(ro, rp, 3)


@pytest.mark.parametrize("pars", [
    # the reference's FFT preconditioner removes segment means and stalls
    # (rr/rrinit ~1e-2 after 200 iterations); compare a bounded run
    dict(use_fprecond=True, iter_max=12),
    dict(precond_width_max=1),
    dict(precond_width_min=0, precond_width_max=0),
    dict(use_cgprecond=True),
    dict(kfilter=False),
    dict(kfilter=False, diagfilter=0.5),
    dict(rm_monopole=True),
    dict(precond_width_min=3, precond_width_max=30),
    dict(mode_detweight=1),
])
def test_solver_options(W, pars):
    d = syn.to_numpy(syn.generate(syn.small_config(seed=21)))
    ro, rp, _, _ = run_both(W, d, pars)
    compare(ro, rp, 3)


def test_cross_resolution_lower_than_map(W):
    d = syn.to_numpy(syn.generate(syn.small_config(seed=22, nside=32)))
    ro, rp, _, _ = run_both(W, d, dict(nside_cross=8, nside_submap=4))
    compare(ro, rp, 3)


def test_write_tod_cleans_signal(W):
    d = syn.to_numpy(syn.generate(syn.small_config(seed=23)))
    ro, rp, do, dp = run_both(W, d, dict(write_tod=True))
    compare(ro, rp, 3)
    _close(dp["signal"], do["signal"], 1e-9)
    assert not np.allclose(dp["signal"], d["signal"])


def test_several_psds_per_detector(W):
    d = syn.to_numpy(syn.generate(syn.small_config(seed=24)))
    ndet = len(d["dets"])
    t0 = d["timestamps"][0]
    mid = d["timestamps"][d["periods"][1]]
    d["npsd"] = np.full(ndet, 2, np.int64)
    d["psdstarts"] = np.tile([t0, mid], ndet)
    base = d["psdvals"].reshape(ndet, -1)
    d["psdvals"] = np.concatenate([np.concatenate([b, 2 * b]) for b in base])
    ro, rp, _, _ = run_both(W, d)
    compare(ro, rp, 3)


def test_device_pointers_match_host_path(W):
    import torch
    cfg = syn.small_config(seed=25)
    dg = syn.generate(cfg, device="cuda")
    dh = syn.to_numpy(dg)
    W.destripe(None, dh["pars"], dh["dets"], dh["detweights"], dh["timestamps"],
               dh["pixels"], dh["pixweights"], dh["signal"], dh["periods"], dh["npsd"],
               dh["psdstarts"], dh["psdfreqs"], dh["psdvals"])
    mh = W.get_result("map")
    W.destripe(None, dg["pars"], dg["dets"], dg["detweights"], dg["timestamps"],
               dg["pixels"].reshape(-1), dg["pixweights"].reshape(-1), dg["signal"].reshape(-1),
               dg["periods"], dg["npsd"], dg["psdstarts"], dg["psdfreqs"], dg["psdvals"])
    torch.cuda.synchronize()
    md = W.get_result("map")
    _close(md, mh, 1e-9)
    np.testing.assert_array_equal(dg["pixels"].cpu().numpy(), dh["pixels"])


def test_pixel_out_of_range_is_an_error(W):
    d = syn.to_numpy(syn.generate(syn.small_config(seed=26)))
    d["pixels"].reshape(-1)[5] = 12 * d["pars"]["nside_map"] ** 2
    with pytest.raises(RuntimeError, match="Too large pixel number"):
        W.destripe(None, d["pars"], d["dets"], d["detweights"], d["timestamps"], d["pixels"],
                   d["pixweights"], d["signal"], d["periods"], d["npsd"], d["psdstarts"],
                   d["psdfreqs"], d["psdvals"])


def test_config1_full_size(W):
    d = syn.to_numpy(syn.generate(syn.config1()))
    ro, rp, _, _ = run_both(W, d)
    compare(ro, rp, 3)


@pytest.mark.parametrize("pars", [
    # invert_pixelmatrix_cross / _map criteria (map_routines.f90:126-182, 255-302):
    # determinant, scaled determinant, rcond, and the cross-only modes 3 / 4
    dict(pixmode_cross=0, pixlim_cross=1e-12, pixmode_map=0, pixlim_map=1e-12),
    dict(pixmode_cross=1, pixlim_cross=1e-3, pixmode_map=1, pixlim_map=1e-3),
    dict(pixmode_cross=3, pixlim_cross=1e-3),
    dict(pixmode_cross=4, pixlim_cross=1e-3),
    dict(pixmode_cross=2, pixlim_cross=0.2, pixmode_map=2, pixlim_map=0.2),
])
def test_pixel_matrix_modes(W, pars):
    d = syn.to_numpy(syn.generate(syn.small_config(seed=27)))
    ro, rp, _, _ = run_both(W, d, pars)
    compare(ro, rp, 3)


def test_good_baseline_fraction(W):
    # flag_bad_baselines (read_data.f90:30-74): without the filter, a baseline
    # with fewer good (unflagged) samples than the fraction loses all of
    # them.  The reference compares the reduced pixel numbers with
    # 12 nside_max^2 (smadam.F90:293), so the rule acts only when every
    # submap is hit: the pointing here is uniform over the sky, a third of
    # the samples flagged (pixel -1)
    d = syn.to_numpy(syn.generate(syn.small_config(seed=28)))
    rng = np.random.default_rng(8)
    n = d["pixels"].size
    npix0 = 12 * d["pars"]["nside_map"] ** 2
    d["pixels"] = rng.integers(0, npix0, d["pixels"].shape).astype(d["pixels"].dtype)
    d["pixels"].reshape(-1)[rng.choice(n, n // 3, replace=False)] = -1
    ro, rp, do, dp = run_both(W, d, dict(kfilter=False, good_baseline_fraction=0.7))
    compare(ro, rp, 3)
    # the rule flags samples (they come back past the dummy pixel,
    # read_data.f90:51 and pointing.f90:178-186) that a run without it keeps
    npix = 12 * d["pars"]["nside_map"] ** 2
    _, _, _, dp0 = run_both(W, d, dict(kfilter=False, good_baseline_fraction=0.0))
    assert (dp["pixels"] >= npix).sum() > (dp0["pixels"] >= npix).sum()


@pytest.mark.parametrize("radiometers", [True, False])
def test_noise_weights_from_psd(W, radiometers):
    # measure_noise_weights (noise_routines.f90:65-127): detector weights from
    # the PSD plateau instead of the caller's detweights
    d = syn.to_numpy(syn.generate(syn.small_config(seed=29)))
    d["detweights"] = d["detweights"] * np.array([0.5, 1.0, 2.0, 4.0])
    ro, rp, _, _ = run_both(W, d, dict(noise_weights_from_psd=True, radiometers=radiometers))
    compare(ro, rp, 3)


def test_checknan_reports_nan_inputs(W, capfd):
    # checknan (smadam_routines.f90:456-502, 978-1033) reports NaNs in the
    # right-hand side and the CG vectors and lets the call go on
    d = syn.to_numpy(syn.generate(syn.small_config(seed=30)))
    pars = dict(d["pars"], checknan=True)
    args = lambda x, s: (pars, x["dets"], x["detweights"], x["timestamps"], x["pixels"].copy(),
                         x["pixweights"], s, x["periods"], x["npsd"], x["psdstarts"],
                         x["psdfreqs"], x["psdvals"])
    W.destripe(None, *args(d, d["signal"].copy()))
    assert not W.get_result("nan_checks").any()
    sig = d["signal"].copy()
    sig.reshape(-1)[1234] = np.nan
    W.destripe(None, *args(d, sig))
    nc = W.get_result("nan_checks")
    assert nc[1] >= 1 and nc[4] >= 1  # yba and r
    out = capfd.readouterr().out
    assert "NaN in uninitialized yba" in out and "r has NaN(s)" in out
