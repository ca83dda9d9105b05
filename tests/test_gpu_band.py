"""The guarded band solve against the state-scan band solve.

The band preconditioner's triangular solves run, by default, as independent
chunks that start their recurrence a checked guard early from a zero state
(band2_solve_guarded); MADAM_B200_BAND_SOLVE=scan selects the exact
chunk-and-state-scan solve instead.  Both apply the same factor, so the
destriped maps, baselines and PCG iteration counts agree to rounding; each
is compared with the CPU oracle elsewhere (test_gpu_parity, test_gpu_shapes).
"""
import numpy as np
import pytest

import parity
from libmadam_b200 import synthetic as syn

pytestmark = pytest.mark.gpu

RTOL = 1e-9  # rounding differences carried through the PCG iterations


@pytest.fixture(scope="module")
def W():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from libmadam_b200 import libmadam_wrapper
    assert libmadam_wrapper.available
    return libmadam_wrapper


def _solve(W, d, pars):
    x = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in d.items()}
    W.destripe(None, pars, x["dets"], x["detweights"], x["timestamps"], x["pixels"],
               x["pixweights"], x["signal"], x["periods"], x["npsd"], x["psdstarts"],
               x["psdfreqs"], x["psdvals"])
    return {k: W.get_result(k) for k in ("map", "aa")} | {"sc": W.scalars()}


@pytest.mark.parametrize("shape", ["plain", "wide", "flagged"])
def test_guarded_matches_scan(W, monkeypatch, shape):
    if shape == "plain":  # the plain float64 workload's per-segment shape
        cfg = syn.config2()
        cfg.ndet, cfg.nobs, cfg.nsamp_obs = 4, 1, 1 << 22
        pars_extra = {}
    else:
        cfg = syn.small_config(seed=81, nsamp_obs=1 << 16, nobs=2)
        pars_extra = dict(precond_width_min=3, precond_width_max=30) if shape == "wide" else {}
    d = syn.to_numpy(syn.generate(cfg, device="cuda"))
    if shape == "flagged":  # nna changes inside the segments
        rng = np.random.default_rng(5)
        n = d["pixels"].size
        d["pixweights"].reshape(-1, 3)[rng.choice(n, n // 20, replace=False)] = 0.0
    pars = dict(d["pars"], **pars_extra)
    monkeypatch.delenv("MADAM_B200_BAND_SOLVE", raising=False)
    g = _solve(W, d, pars)
    monkeypatch.setenv("MADAM_B200_BAND_SOLVE", "scan")
    s = _solve(W, d, pars)
    monkeypatch.delenv("MADAM_B200_BAND_SOLVE")
    assert g["sc"]["band_guard"] > 0 and s["sc"]["band_guard"] == 0
    assert g["sc"]["noiter"] == s["sc"]["noiter"]
    for c in range(3):
        parity.close(g["map"].reshape(-1, 3)[:, c], s["map"].reshape(-1, 3)[:, c], RTOL,
                     "map[%d]" % c)
    parity.close(g["aa"], s["aa"], RTOL, "aa")
