"""Pin the CPU oracle's third-party arithmetic and operator assembly.

The reference links FFTW (r2c/c2r, fourier_fftw_2003.f90:101-123) and LAPACK
(dsyev matrix.f90:102, dpbtrf/dpbtrs noise_routines.f90:1268,1297,
dpotrf/dpotri matrix.f90:297,309).  The oracle restates them; these tests pin
the restatements against numpy.fft (pocketfft) and scipy.linalg.lapack
(OpenBLAS), and pin the destriping operator against a dense numpy build of
A = F^T N^-1 (I - P M P^T N^-1) F + C_a^-1 (Keihanen et al. 2010).
"""
import ctypes as ct

import numpy as np
import pytest
import scipy.linalg.lapack as lapack

import oracle_api as O


def _p(a):
    return a.ctypes.data_as(ct.c_void_p)


@pytest.mark.parametrize("n", [2, 4, 8, 64, 1024, 1 << 15])
def test_rfft_matches_numpy(n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n)
    re = np.empty(n // 2 + 1)
    im = np.empty(n // 2 + 1)
    assert O.lib().oracle_rfft(n, _p(x), _p(re), _p(im)) == 0
    ref = np.fft.rfft(x)
    scale = np.abs(ref).max()
    np.testing.assert_allclose(re, ref.real, atol=1e-13 * scale)
    np.testing.assert_allclose(im, ref.imag, atol=1e-13 * scale)


@pytest.mark.parametrize("n", [2, 4, 16, 4096, 1 << 16])
def test_irfft_matches_numpy(n):
    rng = np.random.default_rng(n + 1)
    X = rng.standard_normal(n // 2 + 1) + 1j * rng.standard_normal(n // 2 + 1)
    out = np.empty(n)
    re = np.ascontiguousarray(X.real)
    im = np.ascontiguousarray(X.imag)
    assert O.lib().oracle_irfft(n, _p(re), _p(im), _p(out)) == 0
    ref = np.fft.irfft(X, n)
    np.testing.assert_allclose(out, ref, atol=1e-14 * np.abs(ref).max())


def test_fft_rejects_non_power_of_two():
    x = np.zeros(12)
    re = np.zeros(7)
    assert O.lib().oracle_rfft(12, _p(x), _p(re), _p(re)) != 0


def _band_spd(n, kd, rng):
    # symmetric Toeplitz band + positive diagonal, like get_cholesky_decomposition
    c = np.exp(-np.arange(kd + 1) / 3.0) * rng.uniform(0.5, 1.0)
    c[0] = 0.0
    diag = rng.uniform(3.0, 5.0, n)
    ab = np.zeros((kd + 1, n))
    for d in range(kd + 1):
        ab[d, :] = c[d]
    ab[0, :] += diag
    return ab


@pytest.mark.parametrize("n,kd", [(1, 0), (5, 2), (200, 9), (1000, 19), (37, 36)])
def test_band_cholesky_matches_lapack(n, kd):
    rng = np.random.default_rng(n * 31 + kd)
    ab = _band_spd(n, kd, rng)
    ref, info = lapack.dpbtrf(ab.copy(), lower=1)
    assert info == 0
    mine = np.ascontiguousarray(ab.T.copy())  # column j contiguous: [j*(kd+1) + d]
    assert O.lib().oracle_pbtrf(n, kd, _p(mine)) == 0
    np.testing.assert_allclose(mine.T, ref, rtol=1e-13, atol=1e-14)
    b = rng.standard_normal(n)
    xref, info = lapack.dpbtrs(ref, b.copy(), lower=1)
    x = b.copy()
    O.lib().oracle_pbtrs(n, kd, _p(mine), _p(x))
    np.testing.assert_allclose(x, xref, rtol=1e-12, atol=1e-14)


def test_band_cholesky_reports_indefinite_column():
    n, kd = 10, 2
    ab = np.zeros((n, kd + 1))
    ab[:, 0] = 1.0
    ab[:, 1] = 2.0  # off-diagonal larger than diagonal -> not positive definite
    info = O.lib().oracle_pbtrf(n, kd, _p(ab))
    _, rinfo = lapack.dpbtrf(np.ascontiguousarray(ab.T.copy()), lower=1)
    assert info == rinfo and info > 0


def test_sym_eig_matches_numpy():
    rng = np.random.default_rng(3)
    for _ in range(200):
        a = rng.standard_normal((3, 3))
        a = a @ a.T + rng.uniform(0, 1) * np.eye(3)
        w = np.empty(3)
        v = np.empty(9)
        af = np.asfortranarray(np.triu(a))  # only the upper triangle is read
        assert O.lib().oracle_sym_eig(3, _p(af), _p(w), _p(v)) == 0
        wr = np.linalg.eigvalsh(a)
        np.testing.assert_allclose(w, wr, rtol=1e-12, atol=1e-14 * wr.max())
        V = v.reshape(3, 3).T
        np.testing.assert_allclose(V @ np.diag(w) @ V.T, a, atol=1e-12 * np.abs(a).max())


@pytest.mark.parametrize("mode", [0, 2])
def test_invert_pixel_matches_numpy(mode):
    rng = np.random.default_rng(11 + mode)
    for _ in range(100):
        a = rng.standard_normal((3, 3))
        a = a @ a.T + 0.5 * np.eye(3)
        cc = np.asfortranarray(np.triu(a)).reshape(-1, order="F").copy()
        crit = ct.c_double()
        sing = O.lib().oracle_invert_pixel(3, mode, _p(cc), ct.byref(crit))
        assert sing == 0
        inv = cc.reshape(3, 3, order="F")
        np.testing.assert_allclose(inv, np.linalg.inv(a), rtol=1e-10, atol=1e-12)
        if mode == 2:
            w = np.linalg.eigvalsh(a)
            assert abs(crit.value - w.min() / w.max()) < 1e-12
        else:
            assert abs(crit.value - np.sqrt(np.linalg.det(a))) < 1e-10 * np.sqrt(np.linalg.det(a))


def test_invert_pixel_singular_is_rejected():
    a = np.zeros(9)
    a[0] = 1.0  # rank one
    crit = ct.c_double()
    assert O.lib().oracle_invert_pixel(3, 2, _p(a), ct.byref(crit)) == 1
    assert np.all(a == 0)


def test_interpolate_psd_loglog():
    f = np.array([0.0, 0.01, 0.1, 1.0, 10.0])
    p = np.array([5.0, 100.0, 10.0, 1.0, 1.0])
    tgt = np.array([0.0, 0.005, 0.01, 0.0316227766, 0.5, 3.0, 10.0, 20.0])
    out = np.empty_like(tgt)
    O.lib().oracle_interpolate_psd(f.size, _p(f), _p(p), tgt.size, _p(tgt), _p(out))
    lf, lp = np.log(f[1:]), np.log(p[1:])

    def ll(x):
        lx = np.log(x)
        j = np.clip(np.searchsorted(lf, lx, side="left") - 1, 0, len(lf) - 2)
        r = (lx - lf[j]) / (lf[j + 1] - lf[j])
        return np.exp(lp[j] * (1 - r) + lp[j + 1] * r)

    assert out[0] == 0.0
    np.testing.assert_allclose(out[1:], [ll(x) for x in tgt[1:]], rtol=1e-12)
