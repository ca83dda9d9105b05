"""The per-pixel tolerance of tests/parity.py on planted errors (numpy, no
GPU): what it accepts and what it must catch."""
import numpy as np
import pytest

import parity as P


def _map(seed=0, n=4096):
    rng = np.random.default_rng(seed)
    b = rng.normal(0, 1e-4, n)
    b[::97] = 0.0                      # unhit pixels
    b[5] = 3e-12                       # a pixel crossing zero, far below the floor
    return b


def test_identical_is_zero():
    b = _map()
    assert P.per_pixel_error(b, b)[0] == 0.0
    assert P.close(b.copy(), b, 1e-6) == 0.0


def test_relative_error_per_pixel():
    b = _map()
    i = int(np.argmax(np.abs(b) > 0.5 * np.abs(b).max()))
    for planted, ok in ((5e-7, True), (2e-6, False)):
        a = b.copy()
        a[i] *= 1 + planted
        e = P.per_pixel_error(a, b)[0]
        assert e == pytest.approx(planted, rel=1e-6)
        if ok:
            P.close(a, b, 1e-6)
        else:
            with pytest.raises(AssertionError):
                P.close(a, b, 1e-6)


def test_a_small_pixel_is_held_to_the_floor_not_to_itself():
    """A value near zero may be off by rtol x floor x max|b| in absolute
    terms, however large that is relative to itself, and not more."""
    b = _map()
    scale = np.abs(b).max()
    a = b.copy()
    a[5] += 0.9e-6 * P.FLOOR * scale   # relative error ~ 1e4 of a 3e-12 value
    P.close(a, b, 1e-6)
    a[5] += 0.2e-6 * P.FLOOR * scale
    with pytest.raises(AssertionError):
        P.close(a, b, 1e-6)


def test_a_pixel_just_above_the_floor_is_relative():
    b = _map()
    scale = np.abs(b).max()
    b[7] = 2 * P.FLOOR * scale
    a = b.copy()
    a[7] *= 1 + 1.5e-6
    with pytest.raises(AssertionError):
        P.close(a, b, 1e-6)


def test_offset_is_removed_only_as_a_constant():
    b = _map()
    nz = b != 0
    a = np.where(nz, b + 3e-5, 0.0)    # the solve's common offset on hit pixels
    with pytest.raises(AssertionError):
        P.close(a, b, 1e-4)
    P.close_modulo_offset(a, b, 1e-6)
    # a planted non-constant error is not absorbed by the offset
    i = int(np.argmax(np.abs(b)))
    a[i] += 1e-3 * abs(b[i])
    with pytest.raises(AssertionError):
        P.close_modulo_offset(a, b, 1e-4)


def test_unhit_pixels_stay_out_of_the_offset():
    """Elements zero in both arrays neither set the offset nor get it."""
    b = _map()
    nz = b != 0
    a = np.where(nz, b - 1e-5, 0.0)
    e, _, _ = P.per_pixel_error_modulo_offset(a, b)
    assert e < 1e-9
    a[~nz] = 1e-9 * np.abs(b).max()    # a value where the reference has none
    e, _, _ = P.per_pixel_error_modulo_offset(a, b)
    assert e > 0


def test_all_zero_reference():
    z = np.zeros(10)
    assert P.per_pixel_error(z, z)[0] == 0.0
    a = z.copy()
    a[3] = 1e-30
    with pytest.raises(AssertionError):
        P.close(a, z, 1e-6)
