"""Drop-in replacement of the reference's Python wrapper.

Same module-level API as python/libmadam_wrapper/__init__.py of the
reference (dtypes 15-19, REPEATED_KEYS 21, dict2parstring 76-88,
dets2detstring 91-98, destripe 101-147, destripe_with_cache 150-172,
clear_caches 175-180), bound to the sm_100a library.  Differences: `comm`
may be None or any object with py2f() (one rank, no MPI); errors raise
RuntimeError instead of aborting the process; array arguments may also be
CUDA tensors / arrays exposing __cuda_array_interface__ (zero-copy, data
stays in HBM).  Results that the reference writes as FITS files are available
from get_result(name).
"""
from __future__ import division, print_function

import ctypes as ct

import numpy as np

from . import _lib

TIMESTAMP_TYPE = np.float64
SIGNAL_TYPE = np.float64
PIXEL_TYPE = np.int32
WEIGHT_TYPE = np.float32
PSD_TYPE = np.float64

REPEATED_KEYS = ["detset", "detset_nopol", "survey"]

try:
    _madam = _lib.load()
except (OSError, RuntimeError):
    _madam = None

available = _madam is not None


def dict2parstring(d):
    """Translate parameter dictionary into a parameter string"""
    s = ""
    for key, value in d.items():
        if key in REPEATED_KEYS:
            for separate_value in value:
                s += "{} = {};".format(key, separate_value)
        else:
            s += "{} = {};".format(key, value)
    return s.encode("ascii")


def dets2detstring(dets):
    """Translate a container of detector names into a detector name string"""
    s = ""
    for d in dets:
        s += "{};".format(d)
    return s.encode("ascii")


def _fcomm(comm):
    """The C-ABI `comm` handle.  None, and any communicator of one rank, run
    one rank (0); a libmadam_b200.comm communicator passes its handle, and an
    int is taken as such a handle.  Any other communicator of several ranks
    (an mpi4py communicator, as the reference wrapper takes) is refused: its
    ranks' reductions would not happen here, so each rank would solve its own
    share of the data alone and write the same file names."""
    if comm is None:
        return 0
    from .comm import _Comm
    if isinstance(comm, _Comm):
        return int(comm.py2f())
    if isinstance(comm, (int, np.integer)):
        return int(comm)
    size = None
    get_size = getattr(comm, "Get_size", None)
    if callable(get_size):
        size = int(get_size())
    elif hasattr(comm, "size"):
        size = int(comm.size)
    if size is not None and size > 1:
        raise ValueError(
            "libmadam_b200: a communicator of {} ranks was passed; sharded runs take a "
            "libmadam_b200.comm.NcclComm or HostComm (this library does not reduce over "
            "MPI)".format(size))
    return 0


class _Buf:
    """A pointer to caller data: host numpy (converted like the reference
    wrapper's np.ascontiguousarray) or a CUDA array passed zero-copy."""

    def __init__(self, a, dtype):
        cai = getattr(a, "__cuda_array_interface__", None)
        if cai is not None:
            if np.dtype(cai["typestr"]) != np.dtype(dtype):
                raise TypeError("device array has dtype {}, expected {}".format(
                    cai["typestr"], np.dtype(dtype)))
            if cai.get("strides") not in (None, ()):
                itemsize = np.dtype(dtype).itemsize
                expect = []
                acc = itemsize
                for n in reversed(cai["shape"]):
                    expect.insert(0, acc)
                    acc *= n
                if tuple(cai["strides"]) != tuple(expect):
                    raise ValueError("device arrays must be C-contiguous")
            self.keep = a
            self.ptr = ct.c_void_p(cai["data"][0])
            self.size = int(np.prod(cai["shape"])) if len(cai["shape"]) else 1
        else:
            arr = np.ascontiguousarray(np.asarray(a).reshape(-1), dtype=dtype)
            self.keep = arr
            self.ptr = arr.ctypes.data_as(ct.c_void_p)
            self.size = arr.size


def _check(status):
    if status != 0:
        _, msg = _lib.last_error()
        raise RuntimeError("libmadam_b200: " + msg)


def destripe(comm, pars, dets, weights, timestamps, pixels, pixweights, signal, periods,
             npsd, psdstarts, psdfreqs, psdvals):
    """
    Solve and subtract baseline offsets from signal
    """
    _destripe(False, comm, pars, dets, weights, timestamps, pixels, pixweights, signal, periods,
              npsd, psdstarts, psdfreqs, psdvals)


def destripe_fp32(comm, pars, dets, weights, timestamps, pixels, pixweights, signal, periods,
                  npsd, psdstarts, psdfreqs, psdvals):
    """
    destripe() on a float32 signal (the FP32-TOD precision form; no
    counterpart in the reference, whose signal is float64): the PCG
    projections read float32 pointing sums and a float32 copy of the map,
    while pixel matrices, baselines and inner products stay float64.  Maps
    and baselines agree with destripe() on the same samples to about 1e-6
    relative.
    """
    _destripe(True, comm, pars, dets, weights, timestamps, pixels, pixweights, signal, periods,
              npsd, psdstarts, psdfreqs, psdvals)


def _destripe(fp32, comm, pars, dets, weights, timestamps, pixels, pixweights, signal, periods,
              npsd, psdstarts, psdfreqs, psdvals):
    if not available:
        raise RuntimeError("No libmadam available, cannot destripe")
    fcomm = _fcomm(comm)
    parstring = dict2parstring(pars)
    ndet = len(dets)
    detstring = dets2detstring(dets)
    ts = _Buf(timestamps, TIMESTAMP_TYPE)
    px = _Buf(pixels, PIXEL_TYPE)
    pw = _Buf(pixweights, WEIGHT_TYPE)
    sg = _Buf(signal, np.float32 if fp32 else SIGNAL_TYPE)
    nsamp = ts.size
    nnz = pw.size // nsamp // ndet
    w = np.ascontiguousarray(weights, dtype=np.float64)
    periods = np.ascontiguousarray(periods, dtype=np.int64)
    npsd = np.ascontiguousarray(npsd, dtype=np.int64)
    psdstarts = np.ascontiguousarray(psdstarts, dtype=np.float64)
    psdfreqs = np.ascontiguousarray(psdfreqs, dtype=np.float64)
    psdvals = np.ascontiguousarray(np.asarray(psdvals).reshape(-1), dtype=PSD_TYPE)
    npsdbin = psdfreqs.size
    npsdval = psdvals.size
    npsdtot = npsdval // npsdbin
    p = lambda a: a.ctypes.data_as(ct.c_void_p)
    entry = _madam.madam_b200_destripe_fp32 if fp32 else _madam.madam_b200_destripe
    status = entry(
        fcomm, parstring, ndet, detstring, p(w), nsamp, nnz, ts.ptr, px.ptr, pw.ptr, sg.ptr,
        periods.size, p(periods), p(npsd), npsdtot, p(psdstarts), npsdbin, p(psdfreqs),
        npsdval, p(psdvals))
    _writeback(pixels, px)
    _writeback(signal, sg)
    _check(status)


def _writeback(orig, buf):
    # the reference mutates the caller's buffers in place when the dtype
    # already matches; mirror that for converted copies too
    if isinstance(orig, np.ndarray) and buf.keep is not orig and orig.size == buf.size:
        if orig.base is not buf.keep and not np.shares_memory(orig, buf.keep):
            try:
                orig.reshape(-1)[:] = buf.keep
            except (ValueError, AttributeError):
                pass


def destripe_with_cache(comm, timestamps, pixels, pixweights, signal, outpath):
    """
    Solve and subtract baseline offsets from signal in Monte Carlo mode
    """
    if not available:
        raise RuntimeError("No libmadam available, cannot destripe")
    fcomm = _fcomm(comm)
    ts = _Buf(timestamps, TIMESTAMP_TYPE)
    px = _Buf(pixels, PIXEL_TYPE)
    pw = _Buf(pixweights, WEIGHT_TYPE)
    sg = _Buf(signal, SIGNAL_TYPE)
    nsamp = ts.size
    ndet = sg.size // nsamp
    nnz = pw.size // nsamp // ndet
    if isinstance(outpath, str):
        outpath = outpath.encode("ascii")
    status = _madam.madam_b200_destripe_with_cache(fcomm, ndet, nsamp, nnz, ts.ptr, px.ptr,
                                                   pw.ptr, sg.ptr, outpath or b"")
    _writeback(pixels, px)
    _writeback(signal, sg)
    _check(status)


def destripe_with_cache_batch(comm, timestamps, pixels, pixweights, signals):
    """
    Batched Monte Carlo: solve every realisation in `signals` ([nrhs, ndet,
    nsamp] or [nrhs, ndet * nsamp]) as destripe_with_cache would right after
    the caching destripe(..., mcmode=True) call, in one multi-right-hand-side
    solve over the shared pointing.  The cache is left unchanged.  Results:
    get_result("map_batch"), "binmap_batch", "aa_batch", "noiter_batch", ...
    (no counterpart in the reference, whose destripe_with_cache takes one
    realisation per call).
    """
    _batch(False, comm, timestamps, pixels, pixweights, signals)


def destripe_with_cache_batch_fp32(comm, timestamps, pixels, pixweights, signals):
    """
    destripe_with_cache_batch on float32 realisations (the FP32-TOD precision
    form): the projections read float32 copies of p.detw and of the map, while
    pixel matrices, baselines and inner products stay float64.  Maps and
    baselines agree with the float64 solve to about 1e-6 relative.
    """
    _batch(True, comm, timestamps, pixels, pixweights, signals)


def _batch(fp32, comm, timestamps, pixels, pixweights, signals):
    if not available:
        raise RuntimeError("No libmadam available, cannot destripe")
    fcomm = _fcomm(comm)
    ts = _Buf(timestamps, TIMESTAMP_TYPE)
    px = _Buf(pixels, PIXEL_TYPE)
    pw = _Buf(pixweights, WEIGHT_TYPE)
    sg = _Buf(signals, np.float32 if fp32 else SIGNAL_TYPE)
    nsamp = ts.size
    ndet = px.size // nsamp
    nnz = pw.size // nsamp // ndet
    nrhs = sg.size // (ndet * nsamp)
    entry = (_madam.madam_b200_destripe_with_cache_batch_fp32 if fp32
             else _madam.madam_b200_destripe_with_cache_batch)
    status = entry(fcomm, ndet, nsamp, nnz, ts.ptr, px.ptr, pw.ptr, nrhs, sg.ptr)
    _writeback(pixels, px)
    _writeback(signals, sg)
    _check(status)


def clear_caches():
    """
    Clear Monte Carlo caches after a destripe() call with mcmode=True
    """
    _check(_madam.madam_b200_clear_caches())


_RESULT_DTYPES = dict(map=np.float64, binmap=np.float64, hits=np.int32, mask=np.int32,
                      crit=np.float32, cc=np.float64, cca=np.float64, aa=np.float64,
                      yba=np.float64, nna=np.float64, fcov=np.float64, invcov=np.float64,
                      rr_history=np.float64, band_widths=np.int64, scalars=np.float64,
                      timings=np.float64, setup_marks=np.float64, map_batch=np.float64,
                      binmap_batch=np.float64, aa_batch=np.float64, noiter_batch=np.float64,
                      rrinit_batch=np.float64, rr_final_batch=np.float64)


def _result_dtype(name):
    if name in _RESULT_DTYPES:
        return _RESULT_DTYPES[name]
    base = name.split("/")[-1]
    ints = ("subset_hits:", "subset_mask:", "subchunk_hits:", "subchunk_mask:")
    if base in ("hits", "mask") or base.startswith(ints):
        return np.int32
    return np.float64


def subsets():
    """The subsets binned by the last call (bin_subsets with detset /
    detset_nopol / survey parameters; smadam.F90:954-1257), in processing
    order: a list of dicts with pass, survey and detset indices (0 = the full
    set), nmap and the result names of its products ("subset_binmap:k" for
    every pass; "subset_hits:k", "subset_mask:k", "subset_cc:k" and, with
    write_leakmatrix, "subset_leak:k:<detector index>" for the first).  The
    full-data leakage matrices are "leakmatrix:<detector index>".  Maps are
    [npix, nmap], matrices [npix, nmap, nmap] (leakage: row i column j)."""
    try:
        tab = get_result("subsets").reshape(-1, 4)
    except KeyError:
        return []
    out = []
    for k, (ps, sv, ds, nm) in enumerate(tab):
        out.append(dict(index=k, pass_=int(ps), survey=int(sv), detset=int(ds), nmap=int(nm),
                        binmap="subset_binmap:%d" % k))
    return out


def get_result(name):
    """Host copy of a result of the last destripe call.

    map / binmap: [npix, nmap] full-sky NESTED maps at nside_map (the values
    the reference writes to *_map.fits / *_bmap.fits); hits, mask, crit:
    [npix]; cc / cca: [npix, nmap, nmap] inverse pixel matrices; aa, yba, nna:
    baselines [ndet, noba]; rr_history: rr/rrinit per PCG iteration.
    """
    L = _lib.load()
    n = L.madam_b200_result_size(name.encode())
    if n < 0:
        raise KeyError(name)
    out = np.empty(n, dtype=_result_dtype(name))
    if n:
        _check(L.madam_b200_result_copy(name.encode(), out.ctypes.data_as(ct.c_void_p),
                                        out.nbytes))
    return out


def scalars():
    keys = ["noiter", "rrinit", "rr_final", "nof", "n_band", "n_band_fail", "iterate_ms",
            "total_ms", "nmap", "noba_short", "npix_map", "nruns", "nwork", "nloc", "nseg",
            "n_cg_prec", "band_rows", "band_transfers", "band_chunks", "scatter_samples",
            "pairs", "fp32", "reliable_updates", "band_guard"]
    return dict(zip(keys, get_result("scalars").tolist()))


def timings():
    keys = ["setup_ms", "iterate_ms", "finalize_ms", "total_ms", "scatter_ms", "gather_ms",
            "filter_ms", "precond_ms", "other_ms"]
    return dict(zip(keys, get_result("timings").tolist()))


def setup_marks():
    """Cumulative host time (ms) after each setup phase of the last destripe:
    input binding (host->device copies), layout (pixel check, periods, baseline
    times), filter, flagging+compaction, runs, binning, pixel-sorted pointing,
    RHS, segments, preconditioner."""
    keys = ["bind", "layout", "filter", "compact", "runs", "bin", "csr", "rhs", "segments",
            "precond"]
    return dict(zip(keys, get_result("setup_marks").tolist()))


def bench_iterations(warmup, iters):
    """Time `iters` PCG iterations (after `warmup`) on the state of the last
    solve, restarted from its right-hand side.  Returns a dict of device
    timings (CUDA events on the library's stream)."""
    out = np.zeros(8)
    _check(_lib.load().madam_b200_bench_iterations(int(warmup), int(iters),
                                                   out.ctypes.data_as(ct.c_void_p), out.size))
    keys = ["total_ms", "ms_per_iter", "launches_per_iter", "scatter_ms", "filter_ms",
            "gather_ms", "precond_ms", "update_ms"]
    return dict(zip(keys, out.tolist()))


def kernel_launches():
    return int(_lib.load().madam_b200_kernel_launches())
