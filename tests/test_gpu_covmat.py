"""The noise covariance files (file_covmat) on the GPU against the oracle:
polarized and temperature-only data, with flagged samples that trim the
pointing periods, files that exist already, and the map left binned (no
solve).  Matrix elements within COV_RTOL of the matrix's largest magnitude:
the GPU sums the pairs of P^T F entries in another order and adds the
white-noise diagonal with FP64 atomics."""
import os

import numpy as np
import pytest

import oracle_api as O
from test_oracle_covmat import _data, read_covmat

pytestmark = pytest.mark.gpu

COV_RTOL = 1e-11


@pytest.fixture(scope="module")
def W():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from libmadam_b200 import libmadam_wrapper
    assert libmadam_wrapper.available
    return libmadam_wrapper


def _args(pars, x):
    return (pars, x["dets"], x["detweights"], x["timestamps"], x["pixels"], x["pixweights"],
            x["signal"], x["periods"], x["npsd"], x["psdstarts"], x["psdfreqs"], x["psdvals"])


def _copy(d):
    return {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in d.items()}


def run_both(W, d, tmp_path, **kw):
    ro, rp = str(tmp_path / "oracle"), str(tmp_path / "gpu")
    O.destripe(*_args(dict(d["pars"], file_covmat=ro, **kw), _copy(d)))
    W.destripe(None, *_args(dict(d["pars"], file_covmat=rp, **kw), _copy(d)))
    return ro, rp


@pytest.mark.parametrize("nnz", [3, 1])
def test_covmat_matches_oracle(W, tmp_path, nnz):
    d = _data(171, nnz)
    ro, rp = run_both(W, d, tmp_path)
    N = 12 * d["pars"]["nside_map"] ** 2 * nnz
    for det in d["dets"]:
        a, b = read_covmat(rp, det, N), read_covmat(ro, det, N)
        np.testing.assert_array_equal(a == -1, b == -1)
        assert np.abs(a - b).max() <= COV_RTOL * np.abs(b).max()
    np.testing.assert_array_equal(W.get_result("hits"), O.result("hits"))
    assert np.all(W.get_result("aa") == 0)
    np.testing.assert_allclose(W.get_result("map"), W.get_result("binmap"), rtol=0, atol=0)


def test_flagged_samples_trim_the_periods(W, tmp_path):
    d = _data(172)
    pix = d["pixels"]
    pix[0, :300] = -1          # the first baselines of a period are empty
    pix[1, 2000:2800] = -1     # a gap longer than a minute splits a period
    pix[0, 5000:5003] = -1
    ro, rp = run_both(W, d, tmp_path)
    N = 12 * d["pars"]["nside_map"] ** 2 * 3
    for det in d["dets"]:
        a, b = read_covmat(rp, det, N), read_covmat(ro, det, N)
        assert np.abs(a - b).max() <= COV_RTOL * np.abs(b).max()


def test_existing_file_is_kept(W, tmp_path):
    d = _data(173)
    root = str(tmp_path / "gpu")
    keep = "{}_{}_inv_bin.dat".format(root, d["dets"][0])
    with open(keep, "wb") as f:
        f.write(b"keep")
    W.destripe(None, *_args(dict(d["pars"], file_covmat=root), _copy(d)))
    assert open(keep, "rb").read() == b"keep"
    other = "{}_{}_inv_bin.dat".format(root, d["dets"][1])
    assert os.path.getsize(other) == (12 * d["pars"]["nside_map"] ** 2 * 3) ** 2 * 8
