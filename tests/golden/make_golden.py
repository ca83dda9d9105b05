"""Regenerate the known-answer fixtures under tests/golden/.

The fixtures restate the inputs and the numpy reference maps of the
reference's own tests (python/tests/test_libmadam.py:86-133 and
python/tests/test_libmadam_mc.py:100-146): nside 8, 1000 samples, 4
temperature-only detectors, pixels = arange % npix, signal = pixel + N(0,1)
with the legacy numpy seed of the reference test, 4 pointing periods, a flat
10-bin PSD.  The expected hit map is hmap[p] += 1 and the expected binned map
is sum(signal) / hits, computed here with plain numpy, independently of both
the oracle and the CUDA library.

Run:  python tests/golden/make_golden.py
"""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def kat_inputs(seed):
    nside = 8
    npix = 12 * nside ** 2
    fsample = 32.5
    nsamp = 1000
    ndet = 4
    np.random.seed(seed)
    timestamps = np.arange(nsamp, dtype=np.float64)
    pixels = (np.arange(ndet * nsamp) % npix).astype(np.int32)
    pixweights = np.ones(ndet * nsamp, dtype=np.float32)
    signal = pixels.astype(np.float64) + np.random.randn(nsamp * ndet)
    signal2 = (pixels % 12).astype(np.float64) + np.random.randn(nsamp * ndet)
    periods = np.array([0, 250, 500, 750], dtype=np.int64)
    npsdbin = 10
    psdfreqs = np.arange(npsdbin) * fsample / npsdbin
    psdvals = np.ones(npsdbin * ndet)
    hmap = np.zeros(npix, dtype=np.int64)
    bmap = np.zeros(npix, dtype=np.float64)
    np.add.at(hmap, pixels, 1)
    np.add.at(bmap, pixels, signal)
    good = hmap != 0
    bmap[good] /= hmap[good]
    return dict(timestamps=timestamps, pixels=pixels, pixweights=pixweights, signal=signal,
                signal2=signal2, periods=periods, psdfreqs=psdfreqs, psdvals=psdvals,
                hmap=hmap, bmap=bmap)


def main():
    np.savez_compressed(os.path.join(HERE, "kat_libmadam.npz"), **kat_inputs(123456))
    np.savez_compressed(os.path.join(HERE, "kat_libmadam_mc.npz"), **kat_inputs(9876543))


if __name__ == "__main__":
    main()
