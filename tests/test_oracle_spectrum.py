"""file_spectrum on the oracle (read_spectrum, noise_routines.f90:505-596;
get_spectrum_file, 600-634).

The file holds "nobins nodetectors", the detector names, their sigmas, then
one row "freq psd_1 .. psd_n" per bin, read as Fortran list-directed input.
The spectrum of a detector is the log-log interpolation of its column,
clamped to the table's ends, used as it stands (no plateau subtraction), and
the file's sigma replaces the detector's (weights 1/sigma^2).  The oracle's
fcov is checked against a numpy statement of that, and its reading against
the format's variants and errors.
"""
import numpy as np
import pytest

import oracle_api as O
from libmadam_b200 import synthetic as syn


def _spec_file_fcov(freq, psd, fsample, nshort, nof, sigma):
    """build_filter with get_spectrum_file, in numpy."""
    fa = fsample / nshort
    lf, ls = np.log(freq), np.log(psd)
    aspec = np.zeros(nof // 2 + 1)
    i = np.arange(nof)
    for k in range(3):
        f = k * fa + i * fa / nof
        with np.errstate(divide="ignore", invalid="ignore"):
            lt = np.log(f)
            kk = np.clip(np.searchsorted(lf, lt, side="left") - 1, 0, len(lf) - 2)
            p = np.clip((lt - lf[kk]) / (lf[kk + 1] - lf[kk]), 0.0, 1.0)
        p = np.where(np.isnan(p), 0.0, p)
        s = np.exp((1 - p) * ls[kk] + p * ls[kk + 1])
        x = np.pi * f / fa
        with np.errstate(divide="ignore", invalid="ignore"):
            g = np.where(x < 1e-30, 1.0, np.sin(x) ** 2 / x ** 2)
        if k == 0:
            aspec[0] = s[0]
        else:
            aspec[0] += 2 * s[0] * g[0]
        ii = np.arange(1, nof // 2 + 1)
        aspec[ii] += s[ii] * g[ii] + s[nof - ii] * g[nof - ii]
    out = np.where(np.abs(aspec) > sigma * float(np.float32(1e-30)), 1.0 / (fa * aspec), 0.0)
    out[0] = 0.0
    return out


def _table(d, nbin=60):
    freq = np.logspace(-4, np.log10(d["pars"]["fsample"] / 2), nbin)
    ndet = len(d["dets"])
    psd = np.stack([2e-6 * (1 + (freq / (0.05 + 0.02 * j)) ** -1.2) for j in range(ndet)], 1)
    sig = 1e-3 * (1 + 0.1 * np.arange(ndet))
    return freq, psd, sig


def _write(path, names, sig, freq, psd, names_per_line=None, sep=" ", dexp=False):
    fmt = (lambda v: ("%.17e" % v).replace("e", "d")) if dexp else (lambda v: "%.17e" % v)
    with open(path, "w") as f:
        f.write("%d %d   trailing words are ignored\n" % (len(freq), len(names)))
        npl = names_per_line or len(names)
        for a in range(0, len(names), npl):
            f.write(sep.join(names[a:a + npl]) + "\n")
        f.write(sep.join(fmt(s) for s in sig) + "\n")
        for b in range(len(freq)):
            f.write(sep.join(fmt(v) for v in [freq[b]] + list(psd[b])) + "\n")


def _run(d, pars):
    do = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in d.items()}
    O.destripe(pars, do["dets"], do["detweights"], do["timestamps"], do["pixels"],
               do["pixweights"], do["signal"], do["periods"], do["npsd"], do["psdstarts"],
               do["psdfreqs"], do["psdvals"])


def test_fcov_from_the_file(tmp_path, capfd):
    d = syn.to_numpy(syn.generate(syn.small_config(seed=91)))
    freq, psd, sig = _table(d)
    # columns in another order than the detectors, with an extra one
    order = [2, 0, 3, 1]
    names = ["%s_x" % d["dets"][j] for j in order] + ["spare"]
    colpsd = np.concatenate([psd[:, order], psd[:, :1] * 3], 1)
    colsig = np.concatenate([sig[order], [9.0]])
    path = tmp_path / "spec.txt"
    _write(path, names, colsig, freq, colpsd, names_per_line=2, sep=", ", dexp=True)
    pars = dict(d["pars"], file_spectrum=str(path))
    _run(d, pars)
    sc = O.scalars()
    nof = int(sc["nof"])
    nshort = int(round(d["pars"]["base_first"] * d["pars"]["fsample"]))
    fc = O.result("fcov").reshape(len(d["dets"]), -1)
    for j in range(len(d["dets"])):
        ref = _spec_file_fcov(freq, psd[:, j], d["pars"]["fsample"], nshort, nof, sig[j])
        np.testing.assert_allclose(fc[j], ref, rtol=1e-12, atol=0)
    out = capfd.readouterr().out
    for j, name in enumerate(d["dets"]):
        assert "%s, SIGMA ==" % name in out
    assert sc["noiter"] > 0


@pytest.mark.parametrize("case, msg", [
    ("header", "is not formatted correctly"),
    ("missing", "not in"),
    ("short", "Failed to read the table from spectrum file"),
    ("sigmas", "Failed to read detector noise levels from spectrum file"),
])
def test_spectrum_file_errors(tmp_path, case, msg):
    d = syn.to_numpy(syn.generate(syn.small_config(seed=92)))
    freq, psd, sig = _table(d)
    names = list(d["dets"])
    path = tmp_path / "spec.txt"
    if case == "missing":
        names[1] = "other"
    _write(path, names, sig, freq, psd)
    text = path.read_text().splitlines()
    if case == "header":
        text[0] = "many columns"
    elif case == "short":
        text = text[:-3]
    elif case == "sigmas":
        text[2] = "1.0 x 2.0 3.0"
    path.write_text("\n".join(text) + "\n")
    with pytest.raises(O.OracleError, match=msg):
        _run(d, dict(d["pars"], file_spectrum=str(path)))


def test_repeat_counts(tmp_path):
    """List-directed repeat counts ("r*c", r copies of c) in the sigmas and
    the table give the file written out in full."""
    d = syn.to_numpy(syn.generate(syn.small_config(seed=93)))
    freq, psd, _ = _table(d)
    ndet = len(d["dets"])
    sig = np.full(ndet, 2e-3)
    psd = np.repeat(psd[:, :1], ndet, 1)  # one spectrum for every detector
    full, short = tmp_path / "full.txt", tmp_path / "short.txt"
    names = list(d["dets"])
    _write(full, names, sig, freq, psd)
    text = full.read_text().splitlines()
    text[2] = "%d*%.17e" % (ndet, sig[0])
    for b in range(len(freq)):
        text[3 + b] = "%.17e %d*%.17e" % (freq[b], ndet, psd[b, 0])
    short.write_text("\n".join(text) + "\n")
    _run(d, dict(d["pars"], file_spectrum=str(full)))
    ref = O.result("fcov")
    _run(d, dict(d["pars"], file_spectrum=str(short)))
    np.testing.assert_array_equal(O.result("fcov"), ref)


@pytest.mark.parametrize("line", ["1.0 / 2.0", "2*", "0*1.0"])
def test_undefined_sigmas_are_refused(tmp_path, line):
    """A slash or a null value leaves items of the READ undefined."""
    d = syn.to_numpy(syn.generate(syn.small_config(seed=94)))
    freq, psd, sig = _table(d)
    path = tmp_path / "spec.txt"
    _write(path, list(d["dets"]), sig, freq, psd)
    text = path.read_text().splitlines()
    text[2] = line + " " + " ".join("%g" % s for s in sig)
    path.write_text("\n".join(text) + "\n")
    with pytest.raises(O.OracleError, match="Failed to read detector noise levels"):
        _run(d, dict(d["pars"], file_spectrum=str(path)))
