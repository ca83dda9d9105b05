"""The reference tests' known answers, checked on the CPU oracle."""
import numpy as np

import kat
import oracle_api as O


class OracleBackend:
    destripe = staticmethod(O.destripe)
    clear_caches = staticmethod(O.clear_caches)

    @staticmethod
    def destripe_with_cache(timestamps, pixels, pixweights, signal, ndet, outpath=b""):
        O.destripe_with_cache(timestamps, pixels, pixweights, signal, ndet)

    @staticmethod
    def result(name):
        return O.result(name)


def test_libmadam_hits_and_binned_map():
    out = kat.run_libmadam_kat(OracleBackend())
    assert len(out) == 2


def test_libmadam_mc_sequence():
    map1, map2, map3 = kat.run_mc_kat(OracleBackend())
    assert np.all(np.isfinite(map1)) and np.all(np.isfinite(map3))


def test_destripe_with_cache_requires_cache():
    O.clear_caches()
    g = kat.load("kat_libmadam_mc.npz")
    try:
        O.destripe_with_cache(g["timestamps"], g["pixels"].copy(), g["pixweights"],
                              g["signal"].copy(), 4)
    except O.OracleError as e:
        assert "empty caches" in str(e)
    else:
        raise AssertionError("expected an error")
