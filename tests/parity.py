"""Per-pixel tolerance shared by the GPU tests.

A map, baseline vector or TOD `a` matches its reference `b` within `rtol`
when every element satisfies

    |a_i - b_i| <= rtol * max(|b_i|, FLOOR * max_j |b_j|)

that is, a relative error of at most `rtol` per pixel (per baseline, per
sample) for every element whose magnitude is at least FLOOR = 1e-3 of the
largest, and an absolute error of at most rtol * FLOOR * max|b| for the
elements closer to zero, whose relative error has no meaning (a Q or U pixel
that happens to cross zero).  The bar is 1e-6 for the float64 path and 1e-4
for the float32-TOD forms.

Two solves that both stop at cglimit differ by the truncation of the solve
itself unless they take the same iterates.  The float64 path runs the
oracle's operations on the same data, so its PCG follows the oracle's
iterates and stops where they stop.  A solve whose projections round to
float32 follows other iterates, and the truncation can be large beside the
1e-3 floor: on a 4-detector scan at nside 1024 the float32-TOD form stopped
at a true float64 residual of 5e-13 (cglimit 1e-12) differs from the
converged solution by up to 0.07 of the 1e-3 floor's scale in a Q pixel,
and even at cglimit 1e-18 by 0.02, where the float64 solve is within 2e-7;
at cglimit 1e-26 both are within 5e-7.  So the float32-TOD forms are
compared with the oracle with both solved to CONVERGED_CGLIMIT = 1e-26,
where the difference is the arithmetic's, at the usual floor.  Where two
solves must stop at a workload's cglimit (a float32 job alone and in the
serving mix, two float32 runs from host and device buffers) the comparison
takes FP32_FLOOR = 1e-2 instead.

The destriping system is singular along one direction: a common offset of
every baseline is a monopole of the temperature map (the noise prior
removes segment means, and the map absorbs a constant), which is why the
reference offers rm_monopole.  A solve leaves that component where its
rounding puts it, so two solves whose operators round differently (a
float32-TOD form against the float64 oracle) differ by a constant in the
baselines and the opposite constant in the I map, at up to ~1e-4 of the
largest baseline and varying from run to run (the setup's float64 atomics
change the last bits of the right-hand side).  close_modulo_offset compares
baselines and I maps with that common constant removed (the mean difference
over the nonzero elements); Q, U and every float64 comparison use close.

With MADAM_PARITY_REPORT=<file> every check appends one JSON line (test,
quantity, error, tolerance, the largest per-element error among the elements
at or above the floor and the absolute error of those below it relative to
max|b|), so a run records the margins as well as the verdicts.
"""
import json
import os

import numpy as np

FLOOR = 1e-3
FP32_FLOOR = 1e-2
CONVERGED_CGLIMIT = 1e-26


def per_pixel_error(a, b, floor=FLOOR):
    """max_i |a_i - b_i| / max(|b_i|, floor * max|b|), with the two parts."""
    a = np.asarray(a, dtype=float).reshape(-1)
    b = np.asarray(b, dtype=float).reshape(-1)
    assert a.shape == b.shape, (a.shape, b.shape)
    if b.size == 0:
        return 0.0, 0.0, 0.0
    mag = np.abs(b)
    scale = float(mag.max())
    diff = np.abs(a - b)
    if scale == 0.0:
        e = float(diff.max()) * 1e300 if diff.max() > 0 else 0.0
        return e, e, 0.0
    cut = floor * scale
    big = mag >= cut
    rel_big = float((diff[big] / mag[big]).max()) if big.any() else 0.0
    abs_small = float(diff[~big].max() / scale) if (~big).any() else 0.0
    return max(rel_big, abs_small / floor), rel_big, abs_small


def close(a, b, rtol, what="", floor=FLOOR):
    """Assert the per-pixel tolerance; returns the error."""
    e, rel_big, abs_small = per_pixel_error(a, b, floor)
    path = os.environ.get("MADAM_PARITY_REPORT")
    if path:
        with open(path, "a") as f:
            f.write(json.dumps({"test": os.environ.get("PYTEST_CURRENT_TEST", "").split(" ")[0],
                                "what": what, "err": e, "rtol": rtol, "floor": floor,
                                "max_rel_above_floor": rel_big,
                                "max_abs_below_floor_over_max": abs_small}) + "\n")
    assert e <= rtol, (what, "per-pixel error", e, "rtol", rtol, rel_big, abs_small)
    return e


def per_pixel_error_modulo_offset(a, b, floor=FLOOR):
    """per_pixel_error after removing the mean of a - b over the elements
    where either is nonzero (the solve's undetermined common offset)."""
    a = np.asarray(a, dtype=float).reshape(-1)
    b = np.asarray(b, dtype=float).reshape(-1)
    nz = (a != 0) | (b != 0)
    off = float(np.mean(a[nz] - b[nz])) if nz.any() else 0.0
    return per_pixel_error(np.where(nz, a - off, a), b, floor)


def close_modulo_offset(a, b, rtol, what="", floor=FLOOR):
    """close() after removing the mean of a - b over the elements where
    either is nonzero (the solve's undetermined common offset)."""
    a = np.asarray(a, dtype=float).reshape(-1)
    b = np.asarray(b, dtype=float).reshape(-1)
    nz = (a != 0) | (b != 0)
    off = float(np.mean(a[nz] - b[nz])) if nz.any() else 0.0
    return close(np.where(nz, a - off, a), b, rtol, what + " (modulo offset %.3g)" % off, floor)
