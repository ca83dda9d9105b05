"""The input mask (file_inmask; read_inmask, read_data.f90:90-190, and the
zeroing of the masked cross-resolution pixel matrices,
map_routines.f90:100-104) on the oracle: a mask that keeps every pixel
changes nothing, a mask that drops pixels zeroes their matrices and changes
the destriped map, and a mask at another resolution is up- or downgraded
to nside_cross."""
import numpy as np
import pytest

import oracle_api as O
from fits_reader import write_mask
from libmadam_b200 import synthetic as syn


def _run(d, pars):
    dd = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in d.items()}
    O.destripe(pars, dd["dets"], dd["detweights"], dd["timestamps"], dd["pixels"],
               dd["pixweights"], dd["signal"], dd["periods"], dd["npsd"], dd["psdstarts"],
               dd["psdfreqs"], dd["psdvals"])
    return {k: O.result(k) for k in ("map", "cca", "aa", "hits")}


def test_keep_all_mask_changes_nothing(tmp_path):
    d = syn.to_numpy(syn.generate(syn.small_config(seed=121)))
    ref = _run(d, d["pars"])
    f = str(tmp_path / "ones.fits")
    write_mask(f, np.ones(12 * 16 ** 2), 16)
    out = _run(d, dict(d["pars"], file_inmask=f))
    for k in ref:
        np.testing.assert_array_equal(out[k], ref[k])


def test_mask_zeroes_cross_matrices_and_up_downgrades(tmp_path):
    d = syn.to_numpy(syn.generate(syn.small_config(seed=122, nside=32)))
    pars = dict(d["pars"], nside_cross=16, nside_submap=4)
    ref = _run(d, pars)
    rng = np.random.default_rng(0)
    m16 = (rng.random(12 * 16 ** 2) > 0.2).astype(float)
    f16 = str(tmp_path / "m16.fits")
    write_mask(f16, m16, 16)
    out16 = _run(d, dict(pars, file_inmask=f16))
    cca = out16["cca"].reshape(-1, 9)
    assert np.all(cca[m16 == 0] == 0)
    assert np.any(cca[m16 == 1] != 0)
    assert not np.allclose(out16["map"], ref["map"])
    np.testing.assert_array_equal(out16["hits"], ref["hits"])
    # the same mask at nside 8 (upgraded) and at nside 32 (downgraded)
    m8 = (rng.random(12 * 8 ** 2) > 0.2).astype(float)
    f8 = str(tmp_path / "m8.fits")
    write_mask(f8, m8, 8, code="D")
    up = _run(d, dict(pars, file_inmask=f8))
    np.testing.assert_array_equal(up["cca"].reshape(-1, 9)[np.repeat(m8, 4) == 0], 0)
    m32 = np.repeat(m16, 4)
    m32[::7] = 0
    f32 = str(tmp_path / "m32.fits")
    write_mask(f32, m32, 32, code="J")
    down = _run(d, dict(pars, file_inmask=f32))
    keep16 = m32.reshape(-1, 4).min(axis=1)
    np.testing.assert_array_equal(down["cca"].reshape(-1, 9)[keep16 == 0], 0)


def test_ring_ordering_is_refused(tmp_path):
    # read_inmask accepts NESTED masks only (read_data.f90:90-190)
    d = syn.to_numpy(syn.generate(syn.small_config(seed=123)))
    f = str(tmp_path / "ring.fits")
    write_mask(f, np.ones(12 * 16 ** 2), 16, ordering="RING")
    with pytest.raises(O.OracleError, match="NESTED"):
        _run(d, dict(d["pars"], file_inmask=f))
