"""FP32-TOD precision form (destripe_fp32) against the FP64 CPU oracle.

The form takes float32 samples and runs the PCG projections on float32
pointing-pair sums and a float32 copy of the map, with pixel matrices,
binning, baselines, inner products and the reliable updates' true residuals
in float64.  The oracle solves the same samples in float64 (the float32
signal widened: identical inputs), and both solve to
parity.CONVERGED_CGLIMIT, so the comparison measures the form's arithmetic,
not the rounding of the input or the truncation of the solve.  Tolerances:
hit counts and masks bit-exact (they do not depend on the signal); binned
maps, destriped maps and baselines within FP32_RTOL per pixel
(parity.close).
"""
import numpy as np
import pytest

import parity
import oracle_api as O
from libmadam_b200 import synthetic as syn

pytestmark = pytest.mark.gpu

FP32_RTOL = 1e-4


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


def _args(pars, x, signal):
    return (pars, x["dets"], x["detweights"], x["timestamps"], x["pixels"], x["pixweights"],
            signal, x["periods"], x["npsd"], x["psdstarts"], x["psdfreqs"], x["psdvals"])


def run_fp32_vs_oracle(W, d, pars=None):
    pars = dict(d["pars"], cglimit=parity.CONVERGED_CGLIMIT, iter_max=2000, **(pars or {}))
    do = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in d.items()}
    dp = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in d.items()}
    sig32 = d["signal"].astype(np.float32)
    do["signal"] = sig32.astype(np.float64)
    O.destripe(*_args(pars, do, do["signal"]))
    ro = {k: O.result(k) for k in ("map", "binmap", "hits", "mask", "aa")}
    ro["scalars"] = O.scalars()
    W.destripe_fp32(None, *_args(pars, dp, sig32))
    rp = {k: W.get_result(k) for k in ("map", "binmap", "hits", "mask", "aa")}
    rp["scalars"] = W.scalars()
    np.testing.assert_array_equal(dp["pixels"], do["pixels"])
    return ro, rp, sig32, do


def compare(ro, rp, nmap):
    np.testing.assert_array_equal(rp["hits"], ro["hits"])
    np.testing.assert_array_equal(rp["mask"], ro["mask"])
    errs = {}
    a = rp["binmap"].reshape(-1, nmap)
    b = ro["binmap"].reshape(-1, nmap)
    errs["binmap"] = max(_close(a[:, c], b[:, c], FP32_RTOL) for c in range(nmap))
    # the destriped I map and the baselines up to the solve's undetermined
    # common offset (parity.close_modulo_offset)
    a = rp["map"].reshape(-1, nmap)
    b = ro["map"].reshape(-1, nmap)
    errs["map"] = max([parity.close_modulo_offset(a[:, 0], b[:, 0], FP32_RTOL, "map[0]")] +
                      [_close(a[:, c], b[:, c], FP32_RTOL) for c in range(1, nmap)])
    errs["aa"] = parity.close_modulo_offset(rp["aa"], ro["aa"], FP32_RTOL, "aa")
    assert rp["scalars"]["fp32"] == 1.0
    return errs


@pytest.mark.parametrize("seed", [7, 8])
def test_fp32_iqu_matches_fp64_oracle(W, seed):
    d = syn.to_numpy(syn.generate(syn.small_config(seed=seed)))
    ro, rp, _, _ = run_fp32_vs_oracle(W, d)
    errs = compare(ro, rp, 3)
    # the projections ran over pointing pairs, fewer than the samples
    sc = rp["scalars"]
    assert 0 < sc["pairs"] < d["pixels"].size
    # float32 projections with reliable updates, both solves converged: the
    # error is far below the tolerance
    assert errs["map"] < 1e-5, errs
    assert sc["noiter"] <= 2.5 * ro["scalars"]["noiter"] + 3  # converges, in more steps
    assert sc["reliable_updates"] >= 1


def test_fp32_temperature_only(W):
    cfg = syn.small_config(seed=11, temperature_only=True)
    d = syn.to_numpy(syn.generate(cfg, nnz=1))
    ro, rp, _, _ = run_fp32_vs_oracle(W, d)
    compare(ro, rp, 1)


@pytest.mark.parametrize("pars", [
    dict(kfilter=False),
    dict(precond_width_min=3, precond_width_max=30),
    dict(nside_cross=8, nside_submap=4),
])
def test_fp32_solver_options(W, pars):
    nside = 32 if "nside_cross" in pars else 16
    d = syn.to_numpy(syn.generate(syn.small_config(seed=31, nside=nside)))
    ro, rp, _, _ = run_fp32_vs_oracle(W, d, pars)
    compare(ro, rp, 3)


def test_fp32_flagged_samples(W):
    d = syn.to_numpy(syn.generate(syn.small_config(seed=32)))
    rng = np.random.default_rng(3)
    n = d["pixels"].size
    bad = rng.choice(n, n // 40, replace=False)
    d["pixweights"].reshape(-1, 3)[bad] = 0.0
    d["pixels"].reshape(-1)[bad[:10]] = -1
    ro, rp, _, _ = run_fp32_vs_oracle(W, d)
    compare(ro, rp, 3)


def test_fp32_write_tod_returns_float32_cleaned_signal(W):
    d = syn.to_numpy(syn.generate(syn.small_config(seed=33)))
    ro, rp, sig32, do = run_fp32_vs_oracle(W, d, dict(write_tod=True))
    compare(ro, rp, 3)
    _close(sig32, do["signal"], FP32_RTOL)
    assert not np.allclose(sig32, d["signal"].astype(np.float32))


def test_fp32_device_buffers_match_host(W):
    import torch
    cfg = syn.small_config(seed=34)
    dg = syn.generate(cfg, device="cuda")
    dh = syn.to_numpy(dg)
    s32 = dh["signal"].astype(np.float32)
    W.destripe_fp32(None, *_args(dh["pars"], dh, s32))
    mh = W.get_result("map")
    W.destripe_fp32(None, dh["pars"], dg["dets"], dg["detweights"], dg["timestamps"],
                    dg["pixels"].reshape(-1), dg["pixweights"].reshape(-1),
                    dg["signal"].reshape(-1).float(), dg["periods"], dg["npsd"],
                    dg["psdstarts"], dg["psdfreqs"], dg["psdvals"])
    torch.cuda.synchronize()
    # the binning's float64 atomic sums make any two runs differ by rounding,
    # which the float32 projections do not damp: the two solves agree to the
    # accuracy the cglimit gives each (measured 7.5e-7 per pixel)
    parity.close(W.get_result("map"), mh, 1e-5, floor=parity.FP32_FLOOR)


def test_fp32_then_fp64_call_uses_fp64_path(W):
    d = syn.to_numpy(syn.generate(syn.small_config(seed=35)))
    pars = dict(d["pars"])
    dp = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in d.items()}
    W.destripe_fp32(None, *_args(pars, dp, d["signal"].astype(np.float32)))
    assert W.scalars()["fp32"] == 1.0
    dp = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in d.items()}
    W.destripe(None, *_args(pars, dp, dp["signal"]))
    sc = W.scalars()
    assert sc["fp32"] == 0.0 and sc["pairs"] == 0.0
