"""Higher-order baselines (basis_order > 0) on the oracle: the basis tables
of start_timeloop (parameter_control.f90:853-933), initialize_a's F^T F
blocks and their inverses (smadam_routines.f90:505-671) and the general
projections of iterate_a (1140-1226, 1379-1480).

Known answers: a sky seen through linear drifts is recovered by first-order
baselines (Legendre or polynomial) to the solver's tolerance, and not by
offsets alone; two bases spanning the same functions (polynomial and
Legendre of one order) give the same destriped map."""
import numpy as np
import pytest

import oracle_api as O
from libmadam_b200 import synthetic as syn


def _drift_data(seed=141, nnz=3, drift=1.0, nside=16, noise=0.0):
    """Random pointing (every pixel crossed by many baselines, so that the
    sky is determined up to the monopole) over a Gaussian sky, no noise,
    plus a linear drift per detector and interval: linear inside every
    baseline."""
    cfg = syn.small_config(seed=seed, temperature_only=(nnz == 1), nside=nside)
    d = syn.to_numpy(syn.generate(cfg, nnz=nnz, with_signal=False))
    rng = np.random.default_rng(seed)
    ndet, nsamp = d["pixels"].shape
    npix = 12 * cfg.nside ** 2
    sky = [rng.normal(0, 1e-4, npix), rng.normal(0, 1e-5, npix), rng.normal(0, 1e-5, npix)]
    pix = rng.integers(0, npix, (ndet, nsamp))
    psi = rng.uniform(0, np.pi, (ndet, nsamp))
    w = np.ones((ndet, nsamp, nnz), np.float32)
    if nnz == 3:
        w[..., 1] = np.cos(2 * psi)
        w[..., 2] = np.sin(2 * psi)
    wd = w.astype(np.float64)
    sig = sky[0][pix]
    if nnz == 3:
        sig = sig + sky[1][pix] * wd[..., 1] + sky[2][pix] * wd[..., 2]
    starts = list(d["periods"]) + [nsamp]
    amp = 1e-4 * drift
    for det in range(ndet):
        for a, b in zip(starts[:-1], starts[1:]):
            t = np.arange(b - a) / (b - a)
            sig[det, a:b] += amp * (rng.normal(0, 5) * t + rng.normal(0, 2))
    if noise:
        sig += rng.normal(0, noise, sig.shape)
    d["pixels"] = np.ascontiguousarray(pix.astype(np.int32))
    d["pixweights"] = np.ascontiguousarray(w)
    d["signal"] = np.ascontiguousarray(sig)
    return d, sky


def _run(d, pars):
    x = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in d.items()}
    O.destripe(pars, x["dets"], x["detweights"], x["timestamps"], x["pixels"], x["pixweights"],
               x["signal"], x["periods"], x["npsd"], x["psdstarts"], x["psdfreqs"], x["psdvals"])
    return {k: O.result(k) for k in ("map", "hits", "aa", "nna")}, x


def _map_error(m, sky, hits, nmap):
    m = m.reshape(-1, nmap)
    good = hits > 0
    err = []
    for c in range(nmap):
        diff = m[good, c] - sky[c][good]
        if c == 0:
            diff = diff - diff.mean()  # the offsets leave the monopole free
        err.append(np.abs(diff).max() / np.abs(sky[c][good]).max())
    return max(err)


@pytest.mark.parametrize("func", ["legendre", "poly"])
def test_linear_drifts_removed_by_first_order(func):
    d, sky = _drift_data()
    base = dict(d["pars"], kfilter=False, iter_max=1000, cglimit=1e-24)
    r1, _ = _run(d, dict(base, basis_order=1, basis_func=func))
    r0, _ = _run(d, dict(base, basis_order=0))
    e1 = _map_error(r1["map"], sky, r1["hits"], 3)
    e0 = _map_error(r0["map"], sky, r0["hits"], 3)
    assert e1 < 1e-8, e1
    assert e0 > 100 * e1, (e0, e1)
    # two amplitudes per baseline, a 2 x 2 block each
    nb = r0["aa"].size
    assert r1["aa"].size == 2 * nb and r1["nna"].size == 4 * nb


def test_temperature_only_drifts():
    d, sky = _drift_data(seed=142, nnz=1)
    base = dict(d["pars"], kfilter=False, iter_max=1000, cglimit=1e-24, basis_order=1)
    r1, _ = _run(d, base)
    assert _map_error(r1["map"], sky, r1["hits"], 1) < 1e-8


def test_polynomial_and_legendre_bases_agree():
    d = syn.to_numpy(syn.generate(syn.small_config(seed=143)))
    base = dict(d["pars"], kfilter=False, iter_max=1000, cglimit=1e-24, basis_order=2)
    rl, _ = _run(d, dict(base, basis_func="legendre"))
    rp, _ = _run(d, dict(base, basis_func="poly"))
    ml, mp = rl["map"].reshape(-1, 3), rp["map"].reshape(-1, 3)
    good = rl["hits"] > 0
    for c in range(3):
        a, b = ml[good, c], mp[good, c]
        if c == 0:
            a, b = a - a.mean(), b - b.mean()
        assert np.abs(a - b).max() < 1e-7 * np.abs(b).max()


def _bin(tod, pix, w, detw, npix):
    """numpy binning: per pixel (sum detw w w^T)^-1 sum detw w tod"""
    nnz = w.shape[-1]
    ww = (w[..., :, None] * w[..., None, :] * detw[:, None, None, None]).reshape(-1, nnz * nnz)
    wt = (w * (tod * detw[:, None])[..., None]).reshape(-1, nnz)
    cc = np.zeros((npix, nnz * nnz))
    b = np.zeros((npix, nnz))
    np.add.at(cc, pix.reshape(-1), ww)
    np.add.at(b, pix.reshape(-1), wt)
    out = np.zeros((npix, nnz))
    good = cc[:, 0] > 0
    out[good] = np.linalg.solve(cc[good].reshape(-1, nnz, nnz), b[good][..., None])[..., 0]
    return out


@pytest.mark.parametrize("func,order", [("fourier", 2), ("chebyshev", 2), ("legendre", 3),
                                        ("poly", 1)])
def test_destriped_map_bins_the_cleaned_tod(func, order):
    # the destriped map is the binned TOD minus the baselines' functions
    # (subtract_baselines_a + makemaps), and clean_tod subtracts the same
    # functions from the TOD
    d, _ = _drift_data(seed=144)
    pars = dict(d["pars"], kfilter=False, basis_order=order, basis_func=func, write_tod=True)
    r, x = _run(d, pars)
    mask = O.result("mask").astype(bool)
    assert not np.allclose(x["signal"], d["signal"])
    npix = mask.size
    m = _bin(x["signal"], d["pixels"], d["pixweights"].astype(np.float64), d["detweights"], npix)
    ref = r["map"].reshape(-1, 3)
    for c in range(3):
        scale = np.abs(ref[mask, c]).max()
        assert np.abs(m[mask, c] - ref[mask, c]).max() < 1e-9 * scale


def test_filter_refused_with_higher_orders():
    d = syn.to_numpy(syn.generate(syn.small_config(seed=145)))
    with pytest.raises(O.OracleError, match="Filter only implemented"):
        _run(d, dict(d["pars"], kfilter=True, basis_order=1))


def _numpy_basis(func, order, n):
    """start_timeloop's tables (parameter_control.f90:865-933) from numpy's
    own polynomials: r at sample centres, dr = 2. / nsamp in single
    precision as the reference divides"""
    dr = float(np.float32(2.0) / np.float32(n))
    r = (0.5 * dr - 1) + np.arange(n) * dr
    out = np.zeros((n, order + 1))
    for o in range(order + 1):
        e = np.zeros(o + 1)
        e[o] = 1
        if func == "poly":
            out[:, o] = r ** o
        elif func == "legendre":
            out[:, o] = np.polynomial.legendre.legval(r, e)
        elif func == "chebyshev":
            # second kind, normalised by (1 - r^2)^(1/4)
            th = np.arccos(r)
            out[:, o] = np.sin((o + 1) * th) / np.sin(th) * (1 - r * r) ** 0.25
        else:
            x = np.arange(n) * np.pi / n
            out[:, o] = np.cos(o * x) if o % 2 == 0 else np.sin((o + 1) * x)
    return out


@pytest.mark.parametrize("func", ["legendre", "poly", "chebyshev", "fourier"])
def test_basis_tables_match_numpy(func):
    d = syn.to_numpy(syn.generate(syn.small_config(seed=146)))
    order = 5
    _run(d, dict(d["pars"], kfilter=False, basis_order=order, basis_func=func))
    for n in (10, 7, 50, 4096):
        t = O.result("basis_table:%d" % n).reshape(n, order + 1)
        np.testing.assert_allclose(t, _numpy_basis(func, order, n), rtol=1e-12, atol=1e-12)
