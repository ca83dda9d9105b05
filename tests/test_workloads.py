"""The benchmark workloads as the synthetic generator defines them: shapes,
noise and solver parameters of the four destripe workloads, and the
sizes derived from them with the reference's own formulas (dnshort =
nint(base_first * fsample), inputparam.f90:63; baselines per interval =
(len - 1) / dnshort + 1, parameter_control.f90:306; submap pixels =
(nside / nside_submap)^2, parameter_control.f90:311-313)."""
import pytest

from libmadam_b200 import synthetic as syn


def _derived(cfg):
    n = cfg.ndet * cfg.nobs * cfg.nsamp_obs
    dnshort = int(round(cfg.base_first * cfg.fsample))
    noba = (cfg.nsamp_obs - 1) // dnshort + 1
    return dict(N=n, dnshort=dnshort, baselines=cfg.ndet * cfg.nobs * noba,
                npix=12 * cfg.nside ** 2, nosubpix=(cfg.nside // cfg.nside_submap) ** 2)


@pytest.mark.parametrize("name, shape, noise, derived", [
    ("config1", dict(nside=64, nside_submap=16, ndet=4, nobs=1, nsamp_obs=1 << 20, fsample=10.0,
                     base_first=1.0, temperature_only=False),
     dict(sigma=1e-3, fknee=0.1, alpha=-1.0, npsdbin=1000),
     dict(N=4 * 2 ** 20, dnshort=10, baselines=4 * 104858, npix=49152, nosubpix=16)),
    ("config2", dict(nside=512, nside_submap=16, ndet=16, nobs=4, nsamp_obs=1 << 23,
                     fsample=100.0, base_first=0.5, temperature_only=False),
     dict(sigma=1e-3, fknee=0.05, alpha=-1.5),
     dict(N=2 ** 29, dnshort=50, baselines=64 * 167773, npix=3145728, nosubpix=1024)),
    ("config3", dict(nside=1024, nside_submap=16, ndet=64, nobs=1, nsamp_obs=1 << 24,
                     fsample=100.0, base_first=1.0, temperature_only=False),
     dict(sigma=1e-3, fknee=0.1, alpha=-1.0),
     dict(N=2 ** 30, dnshort=100, baselines=64 * 167773, npix=12582912, nosubpix=4096)),
    ("config4", dict(nside=512, nside_submap=16, ndet=32, nobs=1, nsamp_obs=1 << 22,
                     fsample=100.0, base_first=1.0, temperature_only=False),
     dict(sigma=1e-3, alpha=-1.0, fknee_range=(0.02, 0.2)),
     dict(N=2 ** 27, dnshort=100, baselines=32 * 41944, npix=3145728, nosubpix=1024)),
])
def test_workload(name, shape, noise, derived):
    cfg = getattr(syn, name)()
    for k, v in {**shape, **noise}.items():
        assert getattr(cfg, k) == v, (name, k)
    assert _derived(cfg) == derived
    pars = syn.pars_for(cfg)
    assert pars["kfilter"] is True and pars["cglimit"] == 1e-12
    assert pars["nside_map"] == cfg.nside and pars["fsample"] == cfg.fsample
    assert pars["base_first"] == cfg.base_first


def test_config1_solver_parameters():
    pars = syn.pars_for(syn.config1())
    assert pars["precond_width_min"] == pars["precond_width_max"] == 20
    assert pars["iter_max"] == 100


def test_config4_detector_knees():
    cfg = syn.config4()
    fk = syn.det_fknee(cfg)
    assert len(fk) == cfg.ndet
    assert (fk >= 0.02).all() and (fk <= 0.2).all() and len(set(fk.tolist())) == cfg.ndet


def test_bench_measures_these_workloads():
    """bench.py's default line runs the nside 512, 16 x 4 x 2^23 workload,
    its precision form the nside 1024, 64 x 2^24 one."""
    import importlib.util
    import os
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(root, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    assert bench.config_for("2")[0] == syn.config2()
    assert bench.config_for("1")[0] == syn.config1()
    assert bench.config_for("3")[0] == syn.config3()


def test_serving_request_mix():
    """The serving stream: 2000 requests, Poisson arrivals at 20 per second,
    nside 128-1024, 2-32 detectors, 2^18-2^24 samples per detector,
    base_first 0.25-2 s, half of them float32 TOD."""
    import importlib.util
    import os

    import numpy as np
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(root, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    specs, arrivals = bench.serve_requests(2000, 20.0, 5005)
    assert len(specs) == 2000 and len(arrivals) == 2000
    assert {s["nside"] for s in specs} == {128, 256, 512, 1024}
    nd = np.array([s["ndet"] for s in specs])
    assert nd.min() == 2 and nd.max() == 32
    ns = np.log2([s["nsamp"] for s in specs])
    assert ns.min() >= 18 and ns.max() < 24 and abs(ns.mean() - 21) < 0.2
    assert {s["base_first"] for s in specs} == {0.25, 0.5, 1.0, 2.0}
    assert abs(np.mean([s["f32"] for s in specs]) - 0.5) < 0.05
    gaps = np.diff(np.concatenate([[0.0], arrivals]))
    assert (gaps > 0).all() and abs(gaps.mean() - 0.05) < 0.005
    assert len({s["seed"] for s in specs}) == 2000
    again, _ = bench.serve_requests(2000, 20.0, 5005)
    assert again == specs
