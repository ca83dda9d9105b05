"""The FITS products (libmadam_b200/csrc/fits.cpp) without a GPU: a harness
(tests/fits_harness.cpp) writes a made-up nside 4 run through the library's
own writer, and the files are checked against the FITS standard's layout
(2880-byte blocks of 80-character ASCII cards, the mandatory keywords of a
binary table in their order) and against the values written, column by
column as the reference names them (output.f90: maps 179-190, mask 838-843,
hits 968, matrices 1085, leakage matrices 1239)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import fits_reader as F

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "libmadam_b200", "csrc")
UNSEEN = np.float32(-1.6375e30)
NPIX = 192


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    d = tmp_path_factory.mktemp("fits")
    exe = str(d / "fits_harness")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", CSRC, os.path.join(HERE, "fits_harness.cpp"),
                    os.path.join(CSRC, "fits.cpp"), os.path.join(CSRC, "params.cpp"), "-o", exe],
                   check=True)
    return exe


def _write(harness, tmp_path, nmap):
    out = tmp_path / ("nmap%d" % nmap)
    out.mkdir()
    subprocess.run([harness, str(out), str(nmap)], check=True)
    return out


def _cards(buf, pos):
    """The cards of one header from pos, and the position after it."""
    cards = []
    while True:
        block = buf[pos:pos + 2880]
        assert len(block) == 2880
        pos += 2880
        for i in range(0, 2880, 80):
            c = block[i:i + 80].decode("ascii")
            assert all(32 <= ord(ch) < 127 for ch in c)
            cards.append(c)
            if c.startswith("END     "):
                assert block[i + 80:].strip(b" ") == b""
                return cards, pos


def _check_layout(path):
    buf = open(path, "rb").read()
    assert len(buf) % 2880 == 0
    prim, pos = _cards(buf, 0)
    assert [c[:8].strip() for c in prim[:3]] == ["SIMPLE", "BITPIX", "NAXIS"]
    assert prim[0][10:30].strip() == "T"
    ext, pos = _cards(buf, pos)
    keys = [c[:8].strip() for c in ext]
    assert keys[:8] == ["XTENSION", "BITPIX", "NAXIS", "NAXIS1", "NAXIS2", "PCOUNT", "GCOUNT",
                        "TFIELDS"]
    hdr, cols = F.read_table(path)
    assert hdr["BITPIX"] == 8 and hdr["NAXIS"] == 2 and hdr["PCOUNT"] == 0
    # the data fill their blocks exactly, zero-padded
    nbytes = hdr["NAXIS1"] * hdr["NAXIS2"]
    assert len(buf) == pos + (nbytes + 2879) // 2880 * 2880
    assert buf[pos + nbytes:].strip(b"\0") == b""
    assert hdr["PIXTYPE"] == "HEALPIX" and hdr["ORDERING"] == "NESTED"
    assert hdr["NSIDE"] == 4 and hdr["FIRSTPIX"] == 0 and hdr["LASTPIX"] == NPIX - 1
    return hdr, cols


@pytest.mark.parametrize("nmap", [1, 3])
def test_products(harness, tmp_path, nmap):
    out = _write(harness, tmp_path, nmap)
    px = np.arange(NPIX)
    mask = px % 5 != 0
    names = ["TEMPERATURE", "Q-POLARISATION", "U-POLARISATION"][:nmap]

    for suffix, sign, step, obj in (("map", 1, 0.25, "madam.map"),
                                    ("bmap", -1, 0.5, "madam.binmap")):
        hdr, cols = _check_layout(out / ("run_%s.fits" % suffix))
        assert hdr["OBJTYPE"] == obj and hdr["POLAR"] == (nmap == 3)
        assert list(cols) == names and hdr["TUNIT1"] == "K_CMB"
        for j, n in enumerate(names):
            want = np.where(mask, np.float32(sign * (px + step * j)), UNSEEN)
            np.testing.assert_array_equal(cols[n], want.astype(np.float32))

    hdr, cols = _check_layout(out / "run_hmap.fits")
    assert hdr["OBJTYPE"] == "madam.hits" and list(cols) == ["Total hits"]
    np.testing.assert_array_equal(cols["Total hits"], 3 * px)

    hdr, cols = _check_layout(out / "run_mask.fits")
    assert list(cols) == ["Mask", "criterion"]
    np.testing.assert_array_equal(cols["Mask"], mask.astype(np.int32))
    np.testing.assert_array_equal(cols["criterion"], (0.5 * px).astype(np.float32))

    # the upper triangle of cc(nmap, nmap, pixel), column-major as in Fortran
    for fname, val in (("wcov_inv", lambda p, k: p + k / 16.0),
                       ("wcov", lambda p, k: 1.0 / (1 + p + k))):
        hdr, cols = _check_layout(out / ("run_%s.fits" % fname))
        assert hdr["OBJTYPE"] == "madam.matrix"
        want_names = ["cc(%d,%d)" % (i + 1, j + 1) for i in range(nmap) for j in range(i, nmap)]
        assert list(cols) == want_names
        for i in range(nmap):
            for j in range(i, nmap):
                np.testing.assert_array_equal(cols["cc(%d,%d)" % (i + 1, j + 1)],
                                              val(px, j * nmap + i))

    hdr, cols = _check_layout(out / "run_leakmatrix_d0.fits")
    assert hdr["OBJTYPE"] == "madam.leakmatrix"
    assert list(cols) == ["gamma(%d,%d)" % (i + 1, j + 1) for i in range(nmap) for j in range(nmap)]
    for i in range(nmap):
        for j in range(nmap):
            np.testing.assert_array_equal(cols["gamma(%d,%d)" % (i + 1, j + 1)],
                                          px * 100.0 + (i * nmap + j))


def test_existing_files(harness, tmp_path):
    """check_outfile (output.f90:1329-1366): an existing file is kept and the
    new one gets the first free "_001".."_999" before its extension; a root
    starting with '!' overwrites instead."""
    out = _write(harness, tmp_path, 1)
    first = sorted(os.listdir(out))
    subprocess.run([harness, str(out), "1"], check=True)
    second = sorted(set(os.listdir(out)) - set(first))
    assert second == sorted(f.replace(".fits", "_001.fits") for f in first)
    subprocess.run([harness, str(out), "1"], check=True)
    assert "run_map_002.fits" in os.listdir(out)
    for f in first:
        assert open(out / f, "rb").read() == open(out / f.replace(".fits", "_001.fits"), "rb").read()
    n = len(os.listdir(out))
    os.remove(out / "run_map.fits")
    subprocess.run([harness, str(out), "1", "!run"], check=True)
    assert len(os.listdir(out)) == n
    _check_layout(out / "run_map.fits")
