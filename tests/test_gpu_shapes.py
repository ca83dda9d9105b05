"""GPU against the CPU oracle at the shapes the benchmarks run.

The other parity tests use small scans (nside <= 64, 10 Hz, baselines of at
most 20 samples).  These cases take the benchmarked workloads' per-segment
shapes at sizes the oracle solves in seconds:

* the plain float64 workload (nside 512, nside_submap 16, 100 Hz,
  base_first 0.5 s, fknee 0.05 Hz, alpha -1.5): 4 detectors x 2^23 samples,
  the full length of one of its observations, so the filter runs at its
  nof = 2^19 and the band preconditioner over its 167,773-baseline segments;
* the precision form (nside 1024, base_first 1 s, float32 TOD):
  4 detectors x 2^22 samples against the float64 oracle on the same
  (float32) samples;
* the batched Monte Carlo form (nside 512, base_first 1 s, per-detector fknee
  in 0.02-0.2 Hz): noise realisations of 4 detectors x 2^20 samples, a
  float64 batch of 8 and a float32 batch of 4, each realisation against the
  oracle's cached solve;
* baselines longer than the warp-chunk gather takes: base_first 5 s and 20 s
  at 100 Hz (500- and 2000-sample baselines, the tiled and the per-baseline
  map-to-baseline kernels).

Tolerances as in the other parity tests, per pixel (parity.close): float64
maps and baselines 1e-6, float32-TOD 1e-4 (both sides solved to
parity.CONVERGED_CGLIMIT, baselines and I map up to the solve's
undetermined common offset, parity.close_modulo_offset); hits and masks
bit-exact.
"""
import numpy as np
import pytest

import oracle_api as O
import parity
from libmadam_b200 import synthetic as syn

pytestmark = pytest.mark.gpu

MAP_RTOL = 1e-6
BIN_RTOL = 1e-10
FP32_RTOL = 1e-4


@pytest.fixture(scope="module")
def W():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from libmadam_b200 import libmadam_wrapper
    assert libmadam_wrapper.available
    return libmadam_wrapper


def _args(pars, x, signal=None):
    return (pars, x["dets"], x["detweights"], x["timestamps"], x["pixels"], x["pixweights"],
            x["signal"] if signal is None else signal, x["periods"], x["npsd"], x["psdstarts"],
            x["psdfreqs"], x["psdvals"])


def _copy(d):
    return {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in d.items()}


def _data(cfg):
    return syn.to_numpy(syn.generate(cfg, device="cuda"))


def _oracle(d, pars):
    do = _copy(d)
    O.destripe(*_args(pars, do))
    r = {k: O.result(k) for k in ("map", "binmap", "hits", "mask", "aa")}
    r["scalars"] = O.scalars()
    r["pixels"] = do["pixels"]
    return r


def _check(rp, ro, nmap, rtol, bin_rtol, floor=parity.FLOOR, offset_free=False):
    # offset_free: the float32-TOD forms, compared up to the solve's
    # undetermined common offset of baselines and I map
    # (parity.close_modulo_offset)
    np.testing.assert_array_equal(rp["hits"], ro["hits"])
    np.testing.assert_array_equal(rp["mask"], ro["mask"])
    for c in range(nmap):
        parity.close(rp["binmap"].reshape(-1, nmap)[:, c], ro["binmap"].reshape(-1, nmap)[:, c],
                     bin_rtol, "binmap[%d]" % c)
        cmp = parity.close_modulo_offset if (offset_free and c == 0) else parity.close
        cmp(rp["map"].reshape(-1, nmap)[:, c], ro["map"].reshape(-1, nmap)[:, c],
            rtol, "map[%d]" % c, floor)
    (parity.close_modulo_offset if offset_free else parity.close)(rp["aa"], ro["aa"], rtol, "aa",
                                                                  floor)


def test_plain_float64_workload_shape(W):
    cfg = syn.config2()
    cfg.ndet, cfg.nobs = 4, 1
    d = _data(cfg)
    ro = _oracle(d, d["pars"])
    dp = _copy(d)
    W.destripe(None, *_args(d["pars"], dp))
    rp = {k: W.get_result(k) for k in ("map", "binmap", "hits", "mask", "aa")}
    sc = W.scalars()
    assert sc["nof"] == ro["scalars"]["nof"] == 1 << 19
    np.testing.assert_array_equal(dp["pixels"], ro["pixels"])
    _check(rp, ro, 3, MAP_RTOL, BIN_RTOL)
    assert sc["noiter"] == ro["scalars"]["noiter"]


def test_precision_form_workload_shape(W):
    cfg = syn.config3()
    cfg.ndet, cfg.nsamp_obs = 4, 1 << 22
    d = _data(cfg)
    sig32 = d["signal"].astype(np.float32)
    d["signal"] = sig32.astype(np.float64)  # the oracle solves the same samples
    pars = dict(d["pars"], cglimit=parity.CONVERGED_CGLIMIT)  # both converged
    ro = _oracle(d, pars)
    dp = _copy(d)
    W.destripe_fp32(None, *_args(pars, dp, sig32))
    rp = {k: W.get_result(k) for k in ("map", "binmap", "hits", "mask", "aa")}
    sc = W.scalars()
    assert sc["fp32"] == 1.0 and sc["pairs"] > 0
    np.testing.assert_array_equal(dp["pixels"], ro["pixels"])
    _check(rp, ro, 3, FP32_RTOL, BIN_RTOL, offset_free=True)
    assert sc["noiter"] <= 2.5 * ro["scalars"]["noiter"] + 3  # converges, in more steps


def _oracle_cached(d, pars, cache_sig, sigs, ndet):
    """The oracle's cached solve of every realisation, each right after the
    caching call (what the batch reproduces)."""
    ref = []
    for s in sigs:
        O.clear_caches()
        do = _copy(d)
        O.destripe(*_args(pars, do, cache_sig.copy()))
        O.destripe_with_cache(d["timestamps"], d["pixels"].copy(), d["pixweights"],
                              s.reshape(-1).copy(), ndet)
        ref.append(dict(map=O.result("map"), aa=O.result("aa"), noiter=O.scalars()["noiter"]))
    O.clear_caches()
    return ref


def test_batched_monte_carlo_workload_shape(W):
    cfg = syn.config4()
    cfg.ndet, cfg.nsamp_obs = 4, 1 << 20
    nrhs = 8
    d = syn.to_numpy(syn.generate(cfg, device="cuda", with_signal=False))
    # realisations that float32 holds exactly, so that the float64 and the
    # float32 batch and the oracle all solve the same samples
    sigs = syn.noise_realisations(cfg, nrhs + 1, device="cuda").float().double().cpu().numpy()
    cache_sig = sigs[nrhs].reshape(-1)
    # float64 batch at the workload's cglimit (it follows the oracle's
    # iterates); float32 batch with both converged (parity.CONVERGED_CGLIMIT)
    cases = ((False, dict(d["pars"], mcmode=True), nrhs),
             (True, dict(d["pars"], mcmode=True, cglimit=parity.CONVERGED_CGLIMIT), 4))
    for fp32, pars, nr in cases:
        ref = _oracle_cached(d, pars, cache_sig, sigs[:nr], cfg.ndet)
        rtol = FP32_RTOL if fp32 else MAP_RTOL
        W.clear_caches()
        W.destripe(None, *_args(pars, _copy(d), cache_sig.copy()))
        if fp32:
            W.destripe_with_cache_batch_fp32(None, d["timestamps"], d["pixels"].copy(),
                                             d["pixweights"], sigs[:nr].astype(np.float32))
        else:
            W.destripe_with_cache_batch(None, d["timestamps"], d["pixels"].copy(),
                                        d["pixweights"], sigs[:nr])
        maps = W.get_result("map_batch").reshape(nr, -1, 3)
        aas = W.get_result("aa_batch").reshape(nr, -1)
        its = W.get_result("noiter_batch")
        for r in range(nr):
            if fp32:
                assert its[r] <= 2.5 * ref[r]["noiter"] + 3  # converges, in more steps
            else:
                assert its[r] == ref[r]["noiter"]
            # the float32 batch up to the solve's undetermined common offset
            # of baselines and I map (parity.close_modulo_offset)
            off = parity.close_modulo_offset if fp32 else parity.close
            for c in range(3):
                (off if c == 0 else parity.close)(maps[r][:, c],
                                                  ref[r]["map"].reshape(-1, 3)[:, c], rtol,
                                                  "map_batch[%d][%d]" % (r, c))
            off(aas[r], ref[r]["aa"], rtol, "aa_batch[%d]" % r)
    W.clear_caches()


@pytest.mark.parametrize("base_first", [5.0, 20.0])
def test_long_baselines(W, base_first):
    cfg = syn.ScanConfig(nside=128, nside_submap=16, ndet=4, nobs=2, nsamp_obs=1 << 19,
                         fsample=100.0, fknee=0.05, alpha=-1.5, base_first=base_first,
                         seed=1200 + int(base_first), extra_pars=dict(cglimit=1e-12))
    d = _data(cfg)
    ro = _oracle(d, d["pars"])
    dp = _copy(d)
    W.destripe(None, *_args(d["pars"], dp))
    rp = {k: W.get_result(k) for k in ("map", "binmap", "hits", "mask", "aa")}
    np.testing.assert_array_equal(dp["pixels"], ro["pixels"])
    _check(rp, ro, 3, MAP_RTOL, BIN_RTOL)
    assert W.scalars()["noiter"] == ro["scalars"]["noiter"]
