"""Subset maps and leakage matrices of the oracle (run_subsets, smadam.F90:
954-1257; leakmatrix, smadam_routines.f90:38-105) against direct numpy
constructions: subset hit maps are counts over the subset's detectors and
time spans, nopol subsets bin the plain TOD mean, polarised subset maps solve
each pixel's 3x3 system, and the leakage matrices of a set's detectors add
up to the identity wherever the set's pixel matrix was inverted."""
import numpy as np

import oracle_api as O
from libmadam_b200 import synthetic as syn


def _data(seed=61):
    cfg = syn.small_config(seed=seed, nsamp_obs=1 << 13)
    return syn.to_numpy(syn.generate(cfg))


def _pars(d):
    t = d["timestamps"]
    mid = t[len(t) // 2]
    return dict(d["pars"], bin_subsets=True, write_leakmatrix=True,
                survey=["hm1 : {} - {}".format(t[0], mid)],
                detset=["AB : det000, det001"], detset_nopol=["CD : det002, det003"])


def _run(d, pars):
    dd = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in d.items()}
    O.destripe(pars, dd["dets"], dd["detweights"], dd["timestamps"], dd["pixels"],
               dd["pixweights"], dd["signal"], dd["periods"], dd["npsd"], dd["psdstarts"],
               dd["psdfreqs"], dd["psdvals"])
    return dd


def test_subset_table_order():
    d = _data()
    _run(d, _pars(d))
    tab = O.result("subsets").reshape(-1, 4)
    # pass 1 only (no binned map requested); survey 0 skips the full set
    assert tab[:, 1:].tolist() == [[0, 1, 3], [0, 2, 1], [1, 0, 3], [1, 1, 3], [1, 2, 1]]


def test_subset_hits_and_maps_match_numpy():
    d = _data()
    pars = _pars(d)
    dd = _run(d, pars)
    npix = 12 * pars["nside_map"] ** 2
    nsamp = d["timestamps"].size
    pix = dd["pixels"].reshape(-1, nsamp)
    w = d["pixweights"].reshape(-1, nsamp, 3).astype(np.float64)
    sig = d["signal"].reshape(-1, nsamp)
    tmask = d["timestamps"] <= d["timestamps"][nsamp // 2]
    tab = O.result("subsets").reshape(-1, 4)
    sets = {0: [0, 1, 2, 3], 1: [0, 1], 2: [2, 3]}
    for k, (_, isv, ids, nmap) in enumerate(tab):
        dets = sets[int(ids)]
        sel = np.zeros(pix.shape, bool)
        sel[dets] = True
        if isv == 1:
            sel &= tmask[None, :]
        sel &= pix < npix
        hits = np.bincount(pix[sel], minlength=npix)
        np.testing.assert_array_equal(O.result("subset_hits:%d" % k), hits)
        mask = O.result("subset_mask:%d" % k)
        bm = O.result("subset_binmap:%d" % k).reshape(npix, int(nmap))
        if nmap == 1:
            s = np.bincount(pix[sel], weights=sig[sel], minlength=npix)
            ref = np.where(hits > 0, s / np.maximum(hits, 1), 0.0)
            np.testing.assert_allclose(bm[:, 0], ref, rtol=1e-10, atol=1e-12)
            continue
        for p in np.flatnonzero(mask > 0)[:200]:
            m = sel & (pix == p)
            A = np.einsum("ni,nj->ij", w[m], w[m])
            b = np.einsum("ni,n->i", w[m], sig[m])
            np.testing.assert_allclose(bm[p], np.linalg.solve(A, b), rtol=1e-6, atol=1e-9)


def test_leakage_matrices_sum_to_identity():
    d = _data()
    pars = _pars(d)
    _run(d, pars)
    npix = 12 * pars["nside_map"] ** 2
    mask = O.result("mask")
    tot = sum(O.result("leakmatrix:%d" % det).reshape(npix, 3, 3) for det in range(4))
    on = mask > 0
    np.testing.assert_allclose(tot[on], np.broadcast_to(np.eye(3), tot[on].shape), atol=1e-8)
    tab = O.result("subsets").reshape(-1, 4)
    sets = {0: [0, 1, 2, 3], 1: [0, 1], 2: [2, 3]}
    for k, (_, isv, ids, nmap) in enumerate(tab):
        nm = int(nmap)
        sm = O.result("subset_mask:%d" % k) > 0
        g = sum(O.result("subset_leak:%d:%d" % (k, det)).reshape(npix, nm, nm)
                for det in sets[int(ids)])
        np.testing.assert_allclose(g[sm], np.broadcast_to(np.eye(nm), g[sm].shape), atol=1e-8)


def test_main_products_unchanged_by_subsets():
    d = _data()
    pars = _pars(d)
    _run(d, dict(d["pars"]))
    ref = {k: O.result(k) for k in ("map", "binmap", "hits", "mask")}
    _run(d, pars)
    for k, v in ref.items():
        np.testing.assert_allclose(O.result(k), v, rtol=1e-12, atol=0)
