"""Backend adapter of the CUDA library for the shared test scenarios."""
import numpy as np

from libmadam_b200 import libmadam_wrapper as W


class ProductBackend:
    @staticmethod
    def destripe(pars, dets, detweights, timestamps, pixels, pixweights, signal, periods, npsd,
                 psdstarts, psdfreqs, psdvals):
        W.destripe(None, pars, dets, detweights, timestamps, pixels, pixweights, signal, periods,
                   npsd, psdstarts, psdfreqs, psdvals)

    @staticmethod
    def destripe_with_cache(timestamps, pixels, pixweights, signal, ndet, outpath=b""):
        W.destripe_with_cache(None, timestamps, pixels, pixweights, signal, outpath)

    @staticmethod
    def clear_caches():
        W.clear_caches()

    @staticmethod
    def result(name):
        r = W.get_result(name)
        return r
