"""Dense numpy restatement of the destriping system, checked against the oracle.

On a tiny problem the whole system can be built explicitly:
  nna_k  = w_d * n_k                                   (initialize_a)
  M      = (P^T N^-1 P)^-1                             (pixel_matrix + invert)
  b      = F^T N^-1 (y - P M P^T N^-1 y)               (initialize_a RHS)
  A      = diag(nna) - F^T N^-1 P M P^T N^-1 F + C_a^-1 (iterate_a A.p)
where C_a^-1 acts per interval as "remove mean, FFT-convolve with fcov,
remove mean" (convolve_interval, noise_routines.f90:816-857) and fcov is the
aliased inverse 1/f spectrum of build_filter (noise_routines.f90:367-739),
restated here in vectorised numpy.  The oracle's RHS, filter and solution must
satisfy these equations.
"""
import numpy as np

import oracle_api as O
from libmadam_b200 import synthetic as syn


def _interp_loglog(freq, psd, target):
    # interpolate_psd (noise_routines.f90:130-190) for ascending targets
    start = np.argmax(freq != 0)
    lf = np.log(np.where(freq > 0, freq, 1.0))
    out = np.zeros_like(target)
    nz = target != 0
    lt = np.log(target[nz])
    j = np.searchsorted(lf[start:], lt, side="left") - 1 + start
    j = np.clip(j, start, len(freq) - 2)
    with np.errstate(divide="ignore", invalid="ignore"):
        r = (lt - lf[j]) / (lf[j + 1] - lf[j])
        logv = np.exp(np.log(psd[j]) * (1 - r) + np.log(psd[j + 1]) * r)
        rl = (target[nz] - freq[j]) / (freq[j + 1] - freq[j])
        lin = psd[j] * (1 - rl) + psd[j + 1] * rl
    out[nz] = np.where((psd[j] > 0) & (psd[j + 1] > 0), logv, lin)
    return out


def _fcov(freqs, psd, fsample, nshort, nof, sigma):
    fa = fsample / nshort
    plateau = _interp_loglog(freqs, psd, np.array([fsample / 2]))[0]
    margin = float(np.float32(1e-6))
    aspec = np.zeros(nof // 2 + 1)
    i = np.arange(nof)
    for k in range(3):
        f = k * fa + i * fa / nof
        s = _interp_loglog(freqs, psd, f)
        s = np.where(s > plateau * (1 + margin), s - plateau, s * margin)
        if f[0] == 0:
            s[0] = 0
        x = np.pi * f / fa
        with np.errstate(divide="ignore", invalid="ignore"):
            g = np.where(x < 1e-30, 1.0, np.sin(x) ** 2 / x ** 2)
        if k == 0:
            aspec[0] = s[0]
        else:
            aspec[0] += 2 * s[0] * g[0]
        ii = np.arange(1, nof // 2 + 1)
        aspec[ii] += s[ii] * g[ii] + s[nof - ii] * g[nof - ii]
    with np.errstate(divide="ignore"):
        out = np.where(np.abs(aspec) > sigma * float(np.float32(1e-30)), 1.0 / (fa * aspec), 0.0)
    out[0] = 0.0
    return out


def _setup():
    cfg = syn.small_config(ndet=3, nsamp_obs=600, nobs=2, nside=2, seed=5,
                           base_first=10.0, fsample=1.0, fknee=0.02)
    cfg.nside_submap = 1
    cfg.extra_pars = dict(iter_max=800, cglimit=1e-26, precond_width_min=3,
                          precond_width_max=8)
    d = syn.to_numpy(syn.generate(cfg))
    return cfg, d


def test_dense_normal_equations():
    cfg, d = _setup()
    ndet, nsamp = cfg.ndet, cfg.nsamp
    pix = d["pixels"].astype(np.int64).copy()
    w = d["pixweights"].astype(np.float64)
    y = d["signal"].copy()
    pixels_in = d["pixels"].copy()
    O.destripe(d["pars"], d["dets"], d["detweights"], d["timestamps"], pixels_in,
               d["pixweights"].copy(), d["signal"].copy(), d["periods"], d["npsd"],
               d["psdstarts"], d["psdfreqs"], d["psdvals"])
    sc = O.scalars()
    nof = int(sc["nof"])
    aa = O.result("aa")
    yba = O.result("yba")
    nna_o = O.result("nna")
    fcov_o = O.result("fcov").reshape(ndet, nof // 2 + 1)
    map_o = O.result("map").reshape(-1, 3)

    npix = 12 * cfg.nside ** 2
    dn = int(round(cfg.base_first * cfg.fsample))
    nper = cfg.nsamp_obs
    nb_int = (nper - 1) // dn + 1
    nbd = nb_int * cfg.nobs
    # sample -> baseline (per detector)
    s = np.arange(nsamp)
    base = (s // nper) * nb_int + (s % nper) // dn
    # detector weights as the reference derives them (1/plateau/fs)
    detw = d["detweights"]
    sig = 1.0 / np.sqrt(detw)
    wd = 1.0 / (sig ** 2 / cfg.fsample) / cfg.fsample
    # pixel matrices and binned map
    cc = np.zeros((npix, 3, 3))
    bm = np.zeros((npix, 3))
    for j in range(ndet):
        np.add.at(cc, pix[j], wd[j] * w[j][:, :, None] * w[j][:, None, :])
        np.add.at(bm, pix[j], wd[j] * w[j] * y[j][:, None])
    M = np.zeros_like(cc)
    for p in range(npix):
        e = np.linalg.eigvalsh(cc[p])
        if e.max() > 0 and e.min() / e.max() >= float(np.float32(1e-3)):
            M[p] = np.linalg.inv(cc[p])
    mbin = np.einsum("pij,pj->pi", M, bm)
    # projection operators as dense matrices
    nb = ndet * nbd
    Z = np.zeros((npix * 3, nb))          # P^T N^-1 F
    for j in range(ndet):
        cols = j * nbd + base
        for c in range(3):
            np.add.at(Z, (pix[j] * 3 + c, cols), wd[j] * w[j][:, c])
    Mbig = np.zeros((npix * 3, npix * 3))
    for p in range(npix):
        Mbig[3 * p:3 * p + 3, 3 * p:3 * p + 3] = M[p]
    # nna and rhs
    nna = np.zeros(nb)
    b = np.zeros(nb)
    for j in range(ndet):
        ok = np.any(M[pix[j]] != 0, axis=(1, 2))
        np.add.at(nna, j * nbd + base[ok], wd[j])
        resid = y[j] - np.einsum("sc,sc->s", w[j], mbin[pix[j]])
        np.add.at(b, j * nbd + base[ok], wd[j] * resid[ok])
    np.testing.assert_allclose(nna_o, nna, rtol=1e-13)
    np.testing.assert_allclose(yba, b, rtol=1e-9, atol=1e-9 * np.abs(b).max())
    # filter
    nshort = dn
    for j in range(ndet):
        fc = _fcov(d["psdfreqs"], d["psdvals"][j * cfg.npsdbin:(j + 1) * cfg.npsdbin],
                   cfg.fsample, nshort, nof, sig[j])
        np.testing.assert_allclose(fcov_o[j], fc, rtol=1e-12)
    Cinv = np.zeros((nb, nb))
    eye = np.eye(nb_int)
    for j in range(ndet):
        kern = np.fft.irfft(fcov_o[j], nof)
        for o in range(cfg.nobs):
            k0 = j * nbd + o * nb_int
            for col in range(nb_int):
                x = eye[col] - eye[col].mean()
                xx = np.zeros(nof)
                xx[:nb_int] = x
                yy = np.fft.irfft(np.fft.rfft(xx) * fcov_o[j], nof)[:nb_int]
                Cinv[k0:k0 + nb_int, k0 + col] = yy - yy.mean()
    A = np.diag(nna) - Z.T @ Mbig @ Z + Cinv
    # solution: equal to the least-squares solution up to the global offset
    res = A @ aa - b
    assert np.linalg.norm(res) < 1e-8 * np.linalg.norm(b)
    x_ls = np.linalg.lstsq(A, b, rcond=1e-13)[0]
    diff = (aa - x_ls) - (aa - x_ls).mean()
    assert np.abs(diff).max() < 1e-6 * np.abs(x_ls).max()
    # destriped map: M P^T N^-1 (y - F a), monopole free
    bm2 = bm - (Z @ aa).reshape(npix, 3)
    map_np = np.einsum("pij,pj->pi", M, bm2)
    hit = np.any(M != 0, axis=(1, 2))
    dm = map_o[hit] - map_np[hit]
    dm[:, 0] -= dm[:, 0].mean()
    assert np.abs(dm).max() < 1e-6 * np.abs(map_np[hit]).max()
