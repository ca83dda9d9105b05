"""The number of pointing weights a sample (nnz) on the oracle.

parameter_control.f90:162-185: nnz = 1 makes the run temperature only;
temperature_only = T with nnz > 1 is refused at the entry point
(smadam.F90:141-144).  nnz other than 1 or 3 is refused as well:
the reference's general pixel-matrix branch (smadam_routines.f90:207-230)
hands its float32 weights (pointing.f90:14) to the float64 BLAS dsyr, so its
result for such nnz is not defined.
"""
import numpy as np
import pytest

import oracle_api as O
from libmadam_b200 import synthetic as syn


def _data(nnz):
    d = syn.to_numpy(syn.generate(syn.small_config(seed=171)))
    w = d["pixweights"]
    ndet, nsamp = d["pixels"].shape
    w = w.reshape(ndet, nsamp, 3)
    extra = [np.full((ndet, nsamp, 1), 0.25, np.float32)] if nnz > 3 else []
    d["pixweights"] = np.ascontiguousarray(
        np.concatenate([w[..., :min(nnz, 3)]] + extra * max(nnz - 3, 0), -1))
    return d


def _run(d, pars):
    do = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in d.items()}
    O.destripe(pars, do["dets"], do["detweights"], do["timestamps"], do["pixels"],
               do["pixweights"], do["signal"], do["periods"], do["npsd"], do["psdstarts"],
               do["psdfreqs"], do["psdvals"])
    return {k: O.result(k) for k in ("map", "binmap", "hits", "aa")}


@pytest.mark.parametrize("nnz", [2, 4])
def test_general_nnz_is_refused(nnz):
    d = _data(nnz)
    with pytest.raises(O.OracleError, match="only nnz = 1 or nnz = 3"):
        _run(d, d["pars"])


@pytest.mark.parametrize("nnz", [2, 3, 4])
def test_temperature_only_with_polarized_weights_is_refused(nnz):
    d = _data(nnz)
    with pytest.raises(O.OracleError, match="temperature_only=T but pointing weights are polarized"):
        _run(d, dict(d["pars"], temperature_only=True))


def test_one_weight_is_temperature_only():
    """nnz = 1 solves for the temperature map whether or not
    temperature_only is set: the same maps, hits and baselines."""
    d = _data(1)
    r0 = _run(d, dict(d["pars"], temperature_only=False))
    r1 = _run(d, dict(d["pars"], temperature_only=True))
    for k in ("map", "binmap", "hits", "aa"):
        np.testing.assert_array_equal(r0[k], r1[k])
    assert r1["map"].size == r1["hits"].size
