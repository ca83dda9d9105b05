"""Known-answer scenarios restated from the reference's own tests.

python/tests/test_libmadam.py:120-174 pins the hit map exactly and the binned
map (allclose) against numpy; python/tests/test_libmadam_mc.py:133-208 adds
the Monte-Carlo cache sequence (mcmode, destripe_with_cache, clear_caches
twice).  The inputs and expected maps live in tests/golden/*.npz
(tests/golden/make_golden.py).  `backend` is any object exposing
destripe / destripe_with_cache / clear_caches / result(name).
"""
import os
import tempfile

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
DETS = ["LFI27M", "LFI27S", "LFI28M", "LFI28S"]


def load(name):
    with np.load(os.path.join(GOLDEN, name)) as z:
        return {k: z[k].copy() for k in z.files}


def libmadam_pars(nside, nside_cross, nside_submap):
    # test_libmadam.py:47-76 (the subset / subchunk keys are added by the caller)
    return {
        "base_first": 1.0, "fsample": 32.5, "nside_map": nside, "nside_cross": nside_cross,
        "nside_submap": nside_submap, "write_map": True, "write_binmap": True,
        "write_matrix": True, "write_wcov": True, "write_hits": True, "kfilter": True,
        "diagfilter": 0, "file_root": "madam_pytest", "iter_max": 100, "allreduce": True,
        "info": 0, "path_output": tempfile.mkdtemp(prefix="madam_kat_"),
    }


def run_libmadam_kat(backend, check_files=False):
    """Two successive destripe() calls with nside_map 8 then 16 (test_libmadam.py:136-153).
    With check_files, the hit and binned maps are also read back from the FITS
    files, as the reference test does with healpy (test_libmadam.py:164-169)."""
    g = load("kat_libmadam.npz")
    nside = 8
    out = []
    nsamp = g["timestamps"].size
    for i in range(2):
        pars = libmadam_pars(nside, 4, 2)
        # the reference test's remaining keys (test_libmadam.py:58-77)
        pars.update(write_leakmatrix=True, nsubchunk=2, bin_subsets=True,
                    survey=["hm1 : {} - {}".format(0, nsamp / 2)])
        pixels = g["pixels"].copy()
        signal = g["signal"].copy()
        backend.destripe(pars, DETS, np.ones(4), g["timestamps"].copy(), pixels,
                         g["pixweights"].copy(), signal, g["periods"], np.ones(4, np.int64),
                         np.zeros(4), g["psdfreqs"], g["psdvals"])
        hits = backend.result("hits")
        binmap = backend.result("binmap")
        npix = 12 * nside ** 2
        assert hits.size == npix
        expect_h = np.zeros(npix, np.int64)
        np.add.at(expect_h, g["pixels"], 1)
        expect_b = np.zeros(npix)
        np.add.at(expect_b, g["pixels"], g["signal"])
        good = expect_h > 0
        expect_b[good] /= expect_h[good]
        if nside == 8:
            np.testing.assert_array_equal(expect_h, g["hmap"])
            np.testing.assert_allclose(expect_b, g["bmap"], rtol=1e-15)
        np.testing.assert_array_equal(hits, expect_h)
        np.testing.assert_allclose(binmap[good], expect_b[good], rtol=1e-12)
        assert np.all(binmap[~good] == 0)
        np.testing.assert_array_equal(pixels, g["pixels"])  # pixels restored
        if check_files:
            from fits_reader import read_table
            hh, hc = read_table(os.path.join(pars["path_output"], "madam_pytest_hmap.fits"))
            assert hh["NSIDE"] == nside and hh["ORDERING"] == "NESTED"
            np.testing.assert_array_equal(hc["Total hits"], expect_h)
            bh, bc = read_table(os.path.join(pars["path_output"], "madam_pytest_bmap.fits"))
            fb = bc["TEMPERATURE"]
            np.testing.assert_allclose(fb[good], expect_b[good].astype(np.float32), rtol=1e-7)
            assert np.all(fb[~good] == np.float32(-1.6375e30))
            mh, mc = read_table(os.path.join(pars["path_output"], "madam_pytest_map.fits"))
            assert mh["OBJTYPE"] == "madam.map"
            np.testing.assert_allclose(mc["TEMPERATURE"][good],
                                       backend.result("map")[good].astype(np.float32), rtol=1e-6)
            for suffix in ("_wcov_inv.fits", "_wcov.fits"):
                assert os.path.exists(os.path.join(pars["path_output"], "madam_pytest" + suffix))
            # the subchunk hit maps add up to the full one (test_libmadam.py:171-174)
            h1 = read_table(os.path.join(pars["path_output"], "madam_pytest_hmap_sub1of2.fits"))
            h2 = read_table(os.path.join(pars["path_output"], "madam_pytest_hmap_sub2of2.fits"))
            np.testing.assert_array_equal(h1[1]["Total hits"] + h2[1]["Total hits"], expect_h)
            assert os.path.exists(os.path.join(pars["path_output"],
                                               "madam_pytest_hm1_hmap_sub1of2.fits"))
        np.testing.assert_array_equal(backend.result("subchunk_hits:1")
                                      + backend.result("subchunk_hits:2"), expect_h)
        out.append((hits, binmap, backend.result("map"), backend.result("aa")))
        nside *= 2
    return out


def run_mc_kat(backend, check_files=False):
    """mcmode cache sequence of test_libmadam_mc.py:133-208; the cached call
    gets an output path as the reference test gives it one
    (test_libmadam_mc.py:173-185), and with check_files its map file is read
    back from there."""
    g = load("kat_libmadam_mc.npz")
    pars = libmadam_pars(8, 8, 8)
    pars["nsubchunk"] = 1
    pars["mcmode"] = False
    del pars["allreduce"]
    args = lambda sig: (pars, DETS, np.ones(4), g["timestamps"].copy(), g["pixels"].copy(),
                        g["pixweights"].copy(), sig, g["periods"], np.ones(4, np.int64),
                        np.zeros(4), g["psdfreqs"], g["psdvals"])
    backend.destripe(*args(g["signal"].copy()))
    hits1 = backend.result("hits")
    bin1 = backend.result("binmap")
    map1 = backend.result("map")
    np.testing.assert_array_equal(hits1, g["hmap"])
    good = g["hmap"] > 0
    np.testing.assert_allclose(bin1[good], g["bmap"][good], rtol=1e-12)
    pars["mcmode"] = True
    backend.destripe(*args(g["signal2"].copy()))
    map2 = backend.result("map")
    outpath = tempfile.mkdtemp(prefix="madam_kat_mc_") + "/"
    backend.destripe_with_cache(g["timestamps"].copy(), g["pixels"].copy(),
                                g["pixweights"].copy(), g["signal"].copy(), 4,
                                outpath.encode("ascii"))
    map3 = backend.result("map")
    if check_files:
        from fits_reader import read_table
        mh, mc = read_table(os.path.join(outpath, "madam_pytest_map.fits"))
        assert mh["OBJTYPE"] == "madam.map"
        good = g["hmap"] > 0
        np.testing.assert_allclose(mc["TEMPERATURE"][good], map3[good].astype(np.float32),
                                   rtol=1e-6)
    backend.clear_caches()
    backend.clear_caches()
    return map1, map2, map3
