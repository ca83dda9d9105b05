"""Serving: jobs of uneven sizes in flight together give the products each
gives alone (same hits and PCG iteration count; maps and baselines within
SERVE_RTOL per pixel: the setup's pixel-matrix and binning scatter sums with
FP64 atomics, so two runs of one job agree to rounding, ~1e-11 after the
PCG, not to the bit), a failing job does not disturb the others, and device
buffers are served like host buffers.  The jobs' PCG iterations run in the
stepper's shared rounds: the job-rounds it counts are the served jobs'
iterations summed, and with several jobs past their setup at once a round
carries more than one job."""
import numpy as np
import pytest

import oracle_api as O
import parity
from libmadam_b200 import synthetic as syn

pytestmark = pytest.mark.gpu

SERVE_RTOL = 1e-9
MAP_RTOL = 1e-6


@pytest.fixture(scope="module")
def W():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from libmadam_b200 import libmadam_wrapper
    return libmadam_wrapper


def _close(a, b, rtol, what=""):
    return parity.close(a, b, rtol, what)


def _jobs():
    specs = [dict(nside=16, ndet=4, nsamp_obs=1 << 14, nobs=2, seed=51),
             dict(nside=32, ndet=2, nsamp_obs=1 << 15, nobs=1, seed=52, base_first=0.5),
             dict(nside=16, ndet=8, nsamp_obs=1 << 13, nobs=3, seed=53, base_first=2.0),
             dict(nside=64, ndet=4, nsamp_obs=1 << 15, nobs=1, seed=54),
             dict(nside=16, ndet=4, nsamp_obs=1 << 14, nobs=1, seed=55, temperature_only=True),
             dict(nside=32, ndet=4, nsamp_obs=1 << 14, nobs=2, seed=56)]
    out = []
    for sp in specs:
        cfg = syn.small_config(**sp)
        out.append(syn.to_numpy(syn.generate(cfg, nnz=1 if sp.get("temperature_only") else None)))
    return out


def _args(d):
    return (d["pars"], d["dets"], d["detweights"], d["timestamps"], d["pixels"].copy(),
            d["pixweights"], d["signal"].copy(), d["periods"], d["npsd"], d["psdstarts"],
            d["psdfreqs"], d["psdvals"])


def test_jobs_in_flight_match_jobs_alone(W):
    from libmadam_b200.serve import Server
    jobs = _jobs()
    alone = []
    for d in jobs:
        W.destripe(None, *_args(d))
        alone.append(dict(map=W.get_result("map"), aa=W.get_result("aa"),
                          hits=W.get_result("hits"), noiter=W.scalars()["noiter"]))
    srv = Server(workers=3, mem_fraction=0.5)
    tickets = [srv.submit(*_args(d)) for d in jobs]
    bad = dict(jobs[0])
    bad_pix = bad["pixels"].copy()
    bad_pix.reshape(-1)[3] = 10 ** 8
    tb = srv.submit(bad["pars"], bad["dets"], bad["detweights"], bad["timestamps"], bad_pix,
                    bad["pixweights"], bad["signal"].copy(), bad["periods"], bad["npsd"],
                    bad["psdstarts"], bad["psdfreqs"], bad["psdvals"])
    served = []
    for t, ref in zip(tickets, alone):
        assert srv.wait(t) == 2
        np.testing.assert_array_equal(srv.result(t, "hits"), ref["hits"])
        _close(srv.result(t, "map"), ref["map"], SERVE_RTOL)
        _close(srv.result(t, "aa"), ref["aa"], SERVE_RTOL)
        assert srv.result(t, "scalars")[0] == ref["noiter"]
        served.append({k: srv.result(t, k) for k in ("map", "aa", "hits")})
        info = srv.info(t)
        assert info["t_end"] >= info["t_start"] >= info["t_submit"]
        srv.release(t)
    # jobs served in the mix against the CPU oracle (the largest, polarised,
    # and the temperature-only job)
    for i, nmap in ((3, 3), (4, 1)):
        O.destripe(*_args(jobs[i]))
        np.testing.assert_array_equal(served[i]["hits"], O.result("hits"))
        mo = O.result("map").reshape(-1, nmap)
        for c in range(nmap):
            _close(served[i]["map"].reshape(-1, nmap)[:, c], mo[:, c], MAP_RTOL, "map[%d]" % c)
        _close(served[i]["aa"], O.result("aa"), MAP_RTOL, "aa")
    with pytest.raises(RuntimeError, match="Too large pixel number"):
        srv.wait(tb)
    st = srv.stats()
    assert st["job_rounds"] == sum(int(a["noiter"]) for a in alone)
    assert st["rounds"] <= st["job_rounds"]
    srv.close()


def test_pcg_rounds_are_shared(W):
    """Four jobs started together: their PCGs share rounds, and each gives
    its lone result."""
    from libmadam_b200.serve import Server
    jobs = [syn.to_numpy(syn.generate(syn.small_config(nside=32, ndet=4, nsamp_obs=1 << 15,
                                                       nobs=2, seed=60 + k)))
            for k in range(4)]
    alone = []
    for d in jobs:
        W.destripe(None, *_args(d))
        alone.append(dict(map=W.get_result("map"), aa=W.get_result("aa"),
                          noiter=W.scalars()["noiter"]))
    srv = Server(workers=4, mem_fraction=0.5)
    tickets = [srv.submit(*_args(d)) for d in jobs]
    for t, ref in zip(tickets, alone):
        assert srv.wait(t) == 2
        assert srv.result(t, "scalars")[0] == ref["noiter"]
        _close(srv.result(t, "map"), ref["map"], SERVE_RTOL)
        _close(srv.result(t, "aa"), ref["aa"], SERVE_RTOL)
    st = srv.stats()
    srv.close()
    assert st["job_rounds"] == sum(int(a["noiter"]) for a in alone)
    assert st["max_jobs"] >= 2 and st["rounds"] < st["job_rounds"], st


def test_device_buffers_are_served(W):
    import torch
    from libmadam_b200.serve import Server
    d = _jobs()[3]
    W.destripe(None, *_args(d))
    ref = W.get_result("map")
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    srv = Server(workers=2)
    t = srv.submit(d["pars"], d["dets"], d["detweights"], dev(d["timestamps"]),
                   dev(d["pixels"]), dev(d["pixweights"]), dev(d["signal"]), d["periods"],
                   d["npsd"], d["psdstarts"], d["psdfreqs"], d["psdvals"])
    assert srv.wait(t) == 2
    _close(srv.result(t, "map"), ref, SERVE_RTOL)
    srv.close()


FP32_RTOL = 1e-4


def test_mixed_float32_and_float64_jobs(W):
    """float32 signals run in the FP32-TOD form (destripe_fp32) and float64
    signals in the float64 form, side by side; each gives its lone result
    (float32 jobs within FP32_RTOL: their float32 projections round the
    setup's rounding-level differences, so two runs agree to ~1e-6)."""
    from libmadam_b200.serve import Server
    jobs = _jobs()
    f32 = [True, False, True, False, True, True]
    alone = []
    for d, f in zip(jobs, f32):
        a = list(_args(d))
        if f:
            a[6] = a[6].astype(np.float32)
            W.destripe_fp32(None, *a)
        else:
            W.destripe(None, *a)
        alone.append(dict(map=W.get_result("map"), aa=W.get_result("aa"),
                          hits=W.get_result("hits"), fp32=W.scalars()["fp32"]))
        assert alone[-1]["fp32"] == (1.0 if f else 0.0)
    srv = Server(workers=3, mem_fraction=0.5)
    tickets = []
    for d, f in zip(jobs, f32):
        a = list(_args(d))
        if f:
            a[6] = a[6].astype(np.float32)
        tickets.append(srv.submit(*a))
    for t, ref, f in zip(tickets, alone, f32):
        assert srv.wait(t) == 2
        np.testing.assert_array_equal(srv.result(t, "hits"), ref["hits"])
        tol = FP32_RTOL if f else SERVE_RTOL
        floor = parity.FP32_FLOOR if f else parity.FLOOR
        parity.close(srv.result(t, "map"), ref["map"], tol, floor=floor)
        parity.close(srv.result(t, "aa"), ref["aa"], tol, floor=floor)
        assert srv.result(t, "scalars")[21] == (1.0 if f else 0.0)
    srv.close()
