"""Batched Monte Carlo solve against one-at-a-time destripe_with_cache calls.

madam_b200_destripe_with_cache_batch solves R noise realisations that share
one pointing as a single multi-right-hand-side PCG.  Each realisation must
come out as destripe_with_cache gives it when called right after the caching
destripe(mcmode=True): same PCG iteration count, destriped and binned maps
and baselines within BATCH_RTOL per pixel (parity.close; the batched
kernels repeat the single-solve arithmetic; the setup's binning scatter sums
with FP64 atomics, so separate runs agree to rounding, not to the bit), and
within MAP_RTOL of the CPU oracle's cached solve of each realisation.
"""
import numpy as np
import pytest

import oracle_api as O
import parity
from libmadam_b200 import synthetic as syn

pytestmark = pytest.mark.gpu

BATCH_RTOL = 1e-9
MAP_RTOL = 1e-6  # against the CPU oracle


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


def _realisations(d, nrhs):
    """Signal plus independent white and 1/f-like noise per realisation."""
    out = []
    for r in range(nrhs):
        rng = np.random.default_rng(1000 + r)
        noise = rng.standard_normal(d["signal"].shape) * 1e-3
        drift = np.cumsum(rng.standard_normal(d["signal"].shape) * 1e-5, axis=-1)
        out.append(d["signal"] + noise + drift)
    return out


def _cache(W, d, pars):
    W.destripe(None, pars, d["dets"], d["detweights"], d["timestamps"], d["pixels"].copy(),
               d["pixweights"], d["signal"].copy(), d["periods"], d["npsd"], d["psdstarts"],
               d["psdfreqs"], d["psdvals"])


def _oracle_sequential(d, pars, sigs):
    """The CPU oracle's cached solve of every realisation, each right after
    the caching call (what the batch reproduces)."""
    res = []
    for s in sigs:
        O.clear_caches()
        O.destripe(pars, d["dets"], d["detweights"], d["timestamps"], d["pixels"].copy(),
                   d["pixweights"], d["signal"].copy(), d["periods"], d["npsd"],
                   d["psdstarts"], d["psdfreqs"], d["psdvals"])
        O.destripe_with_cache(d["timestamps"], d["pixels"].copy(), d["pixweights"], s.copy(),
                              len(d["dets"]))
        res.append({k: O.result(k) for k in ("map", "aa")} | {"noiter": O.scalars()["noiter"]})
    O.clear_caches()
    return res


def _sequential(W, d, pars, sigs):
    res = []
    for s in sigs:
        W.clear_caches()
        _cache(W, d, pars)
        W.destripe_with_cache(None, d["timestamps"], d["pixels"].copy(), d["pixweights"],
                              s.copy(), b"")
        res.append({k: W.get_result(k) for k in ("map", "binmap", "aa")}
                   | {"noiter": W.scalars()["noiter"]})
    return res


@pytest.mark.parametrize("extra", [dict(), dict(temperature_only=True),
                                   dict(precond_width_min=3, precond_width_max=30)])
def test_batch_matches_one_at_a_time(W, extra):
    cfg = syn.small_config(seed=41)
    d = syn.to_numpy(syn.generate(cfg, nnz=1 if extra.get("temperature_only") else None))
    pars = dict(d["pars"], mcmode=True, **extra)
    nrhs = 5
    sigs = _realisations(d, nrhs)
    ref = _sequential(W, d, pars, sigs)
    oref = _oracle_sequential(d, pars, sigs)
    W.clear_caches()
    _cache(W, d, pars)
    W.destripe_with_cache_batch(None, d["timestamps"], d["pixels"].copy(), d["pixweights"],
                                np.stack(sigs))
    nmap = 1 if extra.get("temperature_only") else 3
    maps = W.get_result("map_batch").reshape(nrhs, -1, nmap)
    bins = W.get_result("binmap_batch").reshape(nrhs, -1, nmap)
    aas = W.get_result("aa_batch").reshape(nrhs, -1)
    its = W.get_result("noiter_batch")
    for r in range(nrhs):
        assert its[r] == ref[r]["noiter"] == oref[r]["noiter"]
        for c in range(nmap):
            _close(maps[r][:, c], ref[r]["map"].reshape(-1, nmap)[:, c], BATCH_RTOL)
            _close(bins[r][:, c], ref[r]["binmap"].reshape(-1, nmap)[:, c], BATCH_RTOL)
            _close(maps[r][:, c], oref[r]["map"].reshape(-1, nmap)[:, c], MAP_RTOL,
                   "map_batch vs oracle")
        _close(aas[r], ref[r]["aa"], BATCH_RTOL)
        _close(aas[r], oref[r]["aa"], MAP_RTOL, "aa_batch vs oracle")
    # the cache is left as it was: a following single call gives the sequential answer
    W.destripe_with_cache(None, d["timestamps"], d["pixels"].copy(), d["pixweights"],
                          sigs[2].copy(), b"")
    _close(W.get_result("map").reshape(-1, nmap)[:, 0], ref[2]["map"].reshape(-1, nmap)[:, 0],
           BATCH_RTOL)
    W.clear_caches()


def test_batch_device_buffers(W):
    import torch
    cfg = syn.small_config(seed=43)
    d = syn.to_numpy(syn.generate(cfg))
    pars = dict(d["pars"], mcmode=True)
    sigs = _realisations(d, 3)
    W.clear_caches()
    _cache(W, d, pars)
    W.destripe_with_cache_batch(None, d["timestamps"], d["pixels"].copy(), d["pixweights"],
                                np.stack(sigs))
    mh = W.get_result("map_batch")
    W.clear_caches()
    _cache(W, d, pars)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    W.destripe_with_cache_batch(None, dev(d["timestamps"]), dev(d["pixels"]),
                                dev(d["pixweights"]), dev(np.stack(sigs)))
    torch.cuda.synchronize()
    _close(W.get_result("map_batch"), mh, BATCH_RTOL)
    W.clear_caches()


FP32_RTOL = 1e-4


@pytest.mark.parametrize("extra", [dict(), dict(temperature_only=True)])
def test_batch_fp32_matches_fp64(W, extra):
    """The FP32-TOD batched form against one-at-a-time float64 solves of the
    same samples, both to parity.CONVERGED_CGLIMIT: maps and baselines within
    FP32_RTOL per pixel."""
    cfg = syn.small_config(seed=45)
    d = syn.to_numpy(syn.generate(cfg, nnz=1 if extra.get("temperature_only") else None))
    # both solved to the converged cglimit: the difference is the arithmetic's
    pars = dict(d["pars"], mcmode=True, cglimit=parity.CONVERGED_CGLIMIT, iter_max=2000, **extra)
    nrhs = 4
    # realisations that float32 holds exactly: both sides solve the same data
    sigs = [s.astype(np.float32).astype(np.float64) for s in _realisations(d, nrhs)]
    ref = _sequential(W, d, pars, sigs)
    W.clear_caches()
    _cache(W, d, pars)
    W.destripe_with_cache_batch_fp32(None, d["timestamps"], d["pixels"].copy(), d["pixweights"],
                                     np.stack(sigs).astype(np.float32))
    nmap = 1 if extra.get("temperature_only") else 3
    maps = W.get_result("map_batch").reshape(nrhs, -1, nmap)
    aas = W.get_result("aa_batch").reshape(nrhs, -1)
    its = W.get_result("noiter_batch")
    for r in range(nrhs):
        assert its[r] <= 2.5 * ref[r]["noiter"] + 3  # converges, in more steps
        # up to the solve's undetermined common offset of baselines and I map
        # (parity.close_modulo_offset)
        for c in range(nmap):
            (parity.close_modulo_offset if c == 0 else parity.close)(
                maps[r][:, c], ref[r]["map"].reshape(-1, nmap)[:, c], FP32_RTOL)
        parity.close_modulo_offset(aas[r], ref[r]["aa"], FP32_RTOL)
    # the cache still gives the float64 answer afterwards
    W.destripe_with_cache(None, d["timestamps"], d["pixels"].copy(), d["pixweights"],
                          sigs[1].copy(), b"")
    _close(W.get_result("map").reshape(-1, nmap)[:, 0], ref[1]["map"].reshape(-1, nmap)[:, 0],
           BATCH_RTOL)
    W.clear_caches()
