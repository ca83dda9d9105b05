"""The noise filter's spectra and the preconditioner's band choice on the
GPU against the oracle (build_filter, noise_routines.f90:367-739;
construct_preconditioner, 920-1153).

The spectra are computed on the device from the host's PSD tables and
plateaus; the oracle computes them on the host.  Tolerances: fcov within
1e-12 per bin (parity.close; CUDA's and the C library's log, exp and sin
differ by an ulp), the inverse-covariance kernels within 1e-10 of their
largest magnitude, the band widths equal, maps within 1e-6 and PCG
iteration counts equal.  A PSD with zero values (a spectrum that is not
positive somewhere, which the reference fills from its neighbours) takes the
host's computation, which must give the oracle's spectra to rounding.
"""
import numpy as np
import pytest

import parity
import oracle_api as O
from libmadam_b200 import synthetic as syn
from test_gpu_parity import W, run_both, compare  # noqa: F401

pytestmark = pytest.mark.gpu


def _fcov_check(W, nmap, ro, rp):
    fo = O.result("fcov")
    fp = W.get_result("fcov")
    assert fo.shape == fp.shape
    parity.close(fp, fo, 1e-12, "fcov")
    io = O.result("invcov")
    ip = W.get_result("invcov")
    assert io.shape == ip.shape
    np.testing.assert_allclose(ip, io, rtol=0, atol=1e-10 * np.abs(io).max())
    assert W.scalars()["n_band"] == O.scalars()["n_band_ok"]
    assert W.scalars()["n_band_fail"] == O.scalars()["n_band_fail"]
    compare(ro, rp, nmap)


@pytest.mark.parametrize("extra", [dict(), dict(noise_weights_from_psd=True),
                                   dict(noise_weights_from_psd=True, radiometers=True),
                                   dict(precond_width_min=2, precond_width_max=40)])
def test_device_spectra_match_oracle(W, extra):
    d = syn.to_numpy(syn.generate(syn.small_config(seed=81)))
    ro, rp, _, _ = run_both(W, d, extra)
    _fcov_check(W, 3, ro, rp)


def test_psd_with_zero_bins_takes_the_fill(W):
    d = syn.to_numpy(syn.generate(syn.small_config(seed=82)))
    pv = d["psdvals"].reshape(len(d["dets"]), -1).copy()
    pv[:, 600:620] = 0.0      # zero bins near 0.03 Hz, inside the filter's band
    d["psdvals"] = pv.reshape(-1)
    ro, rp, _, _ = run_both(W, d)
    _fcov_check(W, 3, ro, rp)


def test_file_spectrum_matches_oracle(W, tmp_path):
    # read_spectrum / get_spectrum_file (noise_routines.f90:505-634): the
    # file's spectra and sigmas (columns in another order than the detectors)
    d = syn.to_numpy(syn.generate(syn.small_config(seed=83)))
    ndet = len(d["dets"])
    freq = np.logspace(-4, np.log10(d["pars"]["fsample"] / 2), 80)
    order = list(range(ndet))[::-1]
    with open(tmp_path / "spec.txt", "w") as f:
        f.write("%d %d\n" % (len(freq), ndet))
        f.write(" ".join(d["dets"][j] for j in order) + "\n")
        f.write(" ".join("%.17e" % (1e-3 * (1 + 0.2 * j)) for j in order) + "\n")
        for v in freq:
            f.write("%.17e " % v + " ".join("%.17e" % (3e-6 * (1 + (v / (0.04 + 0.01 * j)) ** -1.5))
                                          for j in order) + "\n")
    ro, rp, _, _ = run_both(W, d, dict(file_spectrum=str(tmp_path / "spec.txt")))
    _fcov_check(W, 3, ro, rp)
