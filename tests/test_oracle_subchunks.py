"""Subchunk passes of the oracle (nsubchunk > 1; smadam.F90:192-437,
parameter_control.f90:820-835): the subchunk hit maps add up to the full hit
map (the reference test's check, test_libmadam.py:171-174), and a subchunk
pass gives what a plain destripe gives with every other sample flagged,
which is how the GPU library runs the passes."""
import numpy as np

import oracle_api as O
from libmadam_b200 import synthetic as syn


def _data(seed=81, **kw):
    cfg = syn.small_config(seed=seed, nsamp_obs=1 << 13, **kw)
    return syn.to_numpy(syn.generate(cfg, nnz=1 if kw.get("temperature_only") else None))


def _run(d, pars, pixels=None):
    dd = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in d.items()}
    if pixels is not None:
        dd["pixels"] = pixels.copy()
    O.destripe(pars, dd["dets"], dd["detweights"], dd["timestamps"], dd["pixels"],
               dd["pixweights"], dd["signal"], dd["periods"], dd["npsd"], dd["psdstarts"],
               dd["psdfreqs"], dd["psdvals"])
    return dd


def _subchunk_of(d, nsub):
    nsamp = d["timestamps"].size
    per = list(d["periods"]) + [nsamp]
    sc = np.zeros(nsamp, int)
    for a, b in zip(per[:-1], per[1:]):
        n = b - a
        sl = n // nsub
        for isub in range(1, nsub + 1):
            lo = a + sl * (isub - 1)
            hi = b if isub == nsub else lo + sl
            sc[lo:hi] = isub
    return sc


def test_subchunk_hits_add_up():
    d = _data()
    _run(d, dict(d["pars"], nsubchunk=3))
    tot = sum(O.result("subchunk_hits:%d" % i) for i in (1, 2, 3))
    np.testing.assert_array_equal(tot, O.result("hits"))


def test_subchunk_pass_equals_flagged_run():
    d = _data(seed=82)
    _run(d, dict(d["pars"], nsubchunk=2))
    sub = {k: O.result("subchunk_%s:2" % k) for k in ("map", "binmap", "hits", "mask")}
    full = {k: O.result(k) for k in ("map", "binmap", "hits")}
    sc = _subchunk_of(d, 2)
    pix = d["pixels"].copy().reshape(-1, sc.size)
    pix[:, sc != 2] = -1
    _run(d, dict(d["pars"]), pixels=pix)
    np.testing.assert_array_equal(O.result("hits"), sub["hits"])
    np.testing.assert_array_equal(O.result("mask"), sub["mask"])
    for k in ("map", "binmap"):
        ref = O.result(k)
        np.testing.assert_allclose(sub[k], ref, rtol=0, atol=1e-10 * np.abs(ref).max())
    # and the full-data pass is the plain destripe
    _run(d, dict(d["pars"]))
    for k, v in full.items():
        np.testing.assert_allclose(v, O.result(k), rtol=0, atol=1e-12 * max(np.abs(v).max(), 1))
