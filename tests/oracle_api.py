"""ctypes binding of the CPU oracle (oracle/liboracle.so) for the test-suite.

The oracle is test infrastructure: only tests/, __graft_entry__.smoke() and
bench.py's CPU legs load it.
"""
import ctypes as ct
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "liboracle.so")

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = ct.CDLL(ORACLE_SO)
        P = ct.c_void_p
        L.oracle_destripe.restype = ct.c_int
        L.oracle_destripe.argtypes = [ct.c_int, ct.c_char_p, ct.c_long, ct.c_char_p, P,
                                      ct.c_long, ct.c_long, P, P, P, P, ct.c_long, P, P,
                                      ct.c_long, P, ct.c_long, P, ct.c_long, P]
        L.oracle_destripe_with_cache.restype = ct.c_int
        L.oracle_destripe_with_cache.argtypes = [ct.c_int, ct.c_long, ct.c_long, ct.c_long,
                                                 P, P, P, P, ct.c_char_p]
        L.oracle_clear_caches.restype = None
        L.oracle_last_error.restype = ct.c_char_p
        L.oracle_result_size.restype = ct.c_long
        L.oracle_result_size.argtypes = [ct.c_char_p]
        L.oracle_result_copy.restype = ct.c_int
        L.oracle_result_copy.argtypes = [ct.c_char_p, P]
        L.oracle_rfft.argtypes = [ct.c_long, P, P, P]
        L.oracle_irfft.argtypes = [ct.c_long, P, P, P]
        L.oracle_pbtrf.argtypes = [ct.c_long, ct.c_long, P]
        L.oracle_pbtrf.restype = ct.c_int
        L.oracle_pbtrs.argtypes = [ct.c_long, ct.c_long, P, P]
        L.oracle_sym_eig.argtypes = [ct.c_int, P, P, P]
        L.oracle_sym_eig.restype = ct.c_int
        L.oracle_invert_pixel.argtypes = [ct.c_int, ct.c_int, P, P]
        L.oracle_invert_pixel.restype = ct.c_int
        L.oracle_interpolate_psd.argtypes = [ct.c_long, P, P, ct.c_long, P, P]
        L.oracle_max_threads.restype = ct.c_int
        L.oracle_set_comm.restype = None
        L.oracle_set_comm.argtypes = [ct.c_int, ct.c_int, ALLREDUCE]
        _lib = L
    return _lib


ALLREDUCE = ct.CFUNCTYPE(None, ct.POINTER(ct.c_double), ct.c_long, ct.c_int)
_comm_keep = []


def set_comm(rank, nranks, allreduce=None):
    """Make the following oracle calls one rank of a sharded run.
    allreduce(array, op) reduces a float64 numpy array in place across the
    ranks (op 0 sum, 1 max); None returns to single-rank runs."""
    L = lib()
    if allreduce is None:
        L.oracle_set_comm(0, 1, ALLREDUCE())
        _comm_keep.clear()
        return

    def cb(ptr, n, op):
        a = np.ctypeslib.as_array(ptr, shape=(n,))
        allreduce(a, op)

    fn = ALLREDUCE(cb)
    _comm_keep[:] = [fn]
    L.oracle_set_comm(rank, nranks, fn)


def _p(a):
    return a.ctypes.data_as(ct.c_void_p)


def dict2parstring(d):
    s = ""
    for key, value in d.items():
        if key in ("detset", "detset_nopol", "survey"):
            for v in value:
                s += "{} = {};".format(key, v)
        else:
            s += "{} = {};".format(key, value)
    return s.encode("ascii")


class OracleError(RuntimeError):
    pass


def destripe(pars, dets, detweights, timestamps, pixels, pixweights, signal, periods,
             npsd, psdstarts, psdfreqs, psdvals):
    """Run the oracle destripe on numpy arrays (pixels / signal mutated in place,
    exactly as the reference mutates the caller's buffers)."""
    L = lib()
    for a, dt in ((timestamps, np.float64), (pixels, np.int32), (pixweights, np.float32),
                  (signal, np.float64)):
        assert a.dtype == dt and a.flags.c_contiguous
    ndet = len(dets)
    nsamp = timestamps.size
    nnz = pixweights.size // nsamp // ndet
    detw = np.ascontiguousarray(detweights, dtype=np.float64)
    periods = np.ascontiguousarray(periods, dtype=np.int64)
    npsd = np.ascontiguousarray(npsd, dtype=np.int64)
    psdstarts = np.ascontiguousarray(psdstarts, dtype=np.float64)
    psdfreqs = np.ascontiguousarray(psdfreqs, dtype=np.float64)
    psdvals = np.ascontiguousarray(psdvals, dtype=np.float64).reshape(-1)
    rc = L.oracle_destripe(0, dict2parstring(pars), ndet, "".join(d + ";" for d in dets).encode(),
                           _p(detw), nsamp, nnz, _p(timestamps), _p(pixels), _p(pixweights),
                           _p(signal), periods.size, _p(periods), _p(npsd), psdvals.size // psdfreqs.size,
                           _p(psdstarts), psdfreqs.size, _p(psdfreqs), psdvals.size, _p(psdvals))
    if rc != 0:
        raise OracleError(L.oracle_last_error().decode())


def destripe_with_cache(timestamps, pixels, pixweights, signal, ndet):
    L = lib()
    nsamp = timestamps.size
    nnz = pixweights.size // nsamp // ndet
    rc = L.oracle_destripe_with_cache(0, ndet, nsamp, nnz, _p(timestamps), _p(pixels),
                                      _p(pixweights), _p(signal), b"")
    if rc != 0:
        raise OracleError(L.oracle_last_error().decode())


def clear_caches():
    lib().oracle_clear_caches()


_DT = dict(map=np.float64, binmap=np.float64, hits=np.int32, mask=np.int32, cc=np.float64,
           cca=np.float64, aa=np.float64, yba=np.float64, nna=np.float64, fcov=np.float64,
           invcov=np.float64, rr_history=np.float64, band_widths=np.int64, scalars=np.float64)


def _dtype(name):
    if name in _DT:
        return _DT[name]
    base = name.split("/")[-1]
    ints = ("subset_hits:", "subset_mask:", "subchunk_hits:", "subchunk_mask:")
    if base in ("hits", "mask") or base.startswith(ints):
        return np.int32
    return np.float64


def result(name):
    L = lib()
    n = L.oracle_result_size(name.encode())
    if n < 0:
        raise KeyError(name)
    out = np.empty(n, dtype=_dtype(name))
    if n:
        L.oracle_result_copy(name.encode(), _p(out))
    return out


def scalars():
    v = result("scalars")
    keys = ["noiter", "rrinit", "rr_final", "nof", "n_band_ok", "n_band_fail", "t_iterate",
            "t_total", "nmap", "noba_short", "nopix_map", "nthreads"]
    return dict(zip(keys, v))
