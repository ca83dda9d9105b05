"""Serving destriping jobs on one GPU (no counterpart in the reference).

    srv = Server(workers=4, mem_fraction=0.8)
    t = srv.submit(pars, dets, weights, timestamps, pixels, pixweights, signal,
                   periods, npsd, psdstarts, psdfreqs, psdvals)
    srv.wait(t)
    m = srv.result(t, "map")
    srv.close()

`submit` takes the arguments of libmadam_wrapper.destripe (the reference's
destripe call without `comm`) and returns at once; a float32 signal runs the
job in the FP32-TOD form of destripe_fp32, any other dtype as float64.  Worker threads, each with
its own engine and CUDA stream, run the jobs; a job starts when its estimated
device footprint fits the memory budget beside the running jobs (first come,
first served), so jobs in flight overlap on the GPU.  The products of a job
are those a lone destripe() call gives.  The ticket keeps the job's buffers
alive until the job is released.
"""
import ctypes as ct

import numpy as np

from . import _lib
from .libmadam_wrapper import (PIXEL_TYPE, PSD_TYPE, SIGNAL_TYPE, TIMESTAMP_TYPE, WEIGHT_TYPE,
                               _Buf, dets2detstring, dict2parstring)

_INT_RESULTS = ("hits", "mask")


def _lib_serve():
    L = _lib.load()
    if getattr(L, "_serve_ready", False):
        return L
    P = ct.c_void_p
    L.madam_b200_serve_open.restype = P
    L.madam_b200_serve_open.argtypes = [ct.c_int, ct.c_double, ct.c_char_p, ct.c_long]
    L.madam_b200_serve_submit.restype = ct.c_long
    L.madam_b200_serve_submit.argtypes = [P, ct.c_char_p, ct.c_long, ct.c_char_p, P, ct.c_long,
                                          ct.c_long, P, P, P, P, ct.c_long, P, P, ct.c_long, P,
                                          ct.c_long, P, ct.c_long, P, ct.c_char_p, ct.c_long]
    L.madam_b200_serve_submit_fp32.restype = ct.c_long
    L.madam_b200_serve_submit_fp32.argtypes = L.madam_b200_serve_submit.argtypes
    L.madam_b200_serve_wait.restype = ct.c_int
    L.madam_b200_serve_wait.argtypes = [P, ct.c_long, ct.c_double]
    L.madam_b200_serve_result_size.restype = ct.c_long
    L.madam_b200_serve_result_size.argtypes = [P, ct.c_long, ct.c_char_p]
    L.madam_b200_serve_result_copy.restype = ct.c_int
    L.madam_b200_serve_result_copy.argtypes = [P, ct.c_long, ct.c_char_p, P, ct.c_long]
    L.madam_b200_serve_job_info.restype = ct.c_int
    L.madam_b200_serve_job_info.argtypes = [P, ct.c_long, P, ct.c_long]
    L.madam_b200_serve_error.restype = ct.c_int
    L.madam_b200_serve_error.argtypes = [P, ct.c_long, ct.c_char_p, ct.c_long]
    L.madam_b200_serve_release.restype = ct.c_int
    L.madam_b200_serve_release.argtypes = [P, ct.c_long]
    L.madam_b200_serve_stats.restype = ct.c_int
    L.madam_b200_serve_stats.argtypes = [P, P, ct.c_long]
    L.madam_b200_serve_close.restype = ct.c_int
    L.madam_b200_serve_close.argtypes = [P]
    L._serve_ready = True
    return L


def _is_float32(a):
    cai = getattr(a, "__cuda_array_interface__", None)
    if cai is not None:
        return np.dtype(cai["typestr"]) == np.float32
    return np.asarray(a).dtype == np.float32


class Ticket:
    """A submitted job: its id and the buffers it reads."""

    def __init__(self, job, keep):
        self.job = job
        self._keep = keep


class Server:
    def __init__(self, workers=4, mem_fraction=0.8):
        self._L = _lib_serve()
        err = ct.create_string_buffer(512)
        self._h = self._L.madam_b200_serve_open(int(workers), float(mem_fraction), err, 512)
        if not self._h:
            raise RuntimeError("libmadam_b200 serve: " + err.value.decode())

    def submit(self, pars, dets, weights, timestamps, pixels, pixweights, signal, periods, npsd,
               psdstarts, psdfreqs, psdvals):
        parstring = dict2parstring(pars)
        ndet = len(dets)
        detstring = dets2detstring(dets)
        ts = _Buf(timestamps, TIMESTAMP_TYPE)
        px = _Buf(pixels, PIXEL_TYPE)
        pw = _Buf(pixweights, WEIGHT_TYPE)
        fp32 = _is_float32(signal)
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
        p = lambda a: a.ctypes.data_as(ct.c_void_p)
        err = ct.create_string_buffer(512)
        entry = self._L.madam_b200_serve_submit_fp32 if fp32 else self._L.madam_b200_serve_submit
        job = entry(
            self._h, parstring, ndet, detstring, p(w), nsamp, nnz, ts.ptr, px.ptr, pw.ptr, sg.ptr,
            periods.size, p(periods), p(npsd), npsdval // npsdbin, p(psdstarts), npsdbin,
            p(psdfreqs), npsdval, p(psdvals), err, 512)
        if job < 0:
            raise RuntimeError("libmadam_b200 serve: " + err.value.decode())
        return Ticket(job, (ts, px, pw, sg, w, periods, npsd, psdstarts, psdfreqs, psdvals,
                            pixels, signal))

    def wait(self, ticket, timeout=None):
        """Job state after waiting: 2 done, 3 failed (raises), 0/1 still pending."""
        st = self._L.madam_b200_serve_wait(self._h, ticket.job,
                                           -1.0 if timeout is None else float(timeout))
        if st == 3:
            buf = ct.create_string_buffer(4096)
            self._L.madam_b200_serve_error(self._h, ticket.job, buf, 4096)
            raise RuntimeError("libmadam_b200 serve job {}: {}".format(ticket.job,
                                                                     buf.value.decode()))
        return st

    def result(self, ticket, name):
        n = self._L.madam_b200_serve_result_size(self._h, ticket.job, name.encode())
        if n < 0:
            raise KeyError("no result {} for job {}".format(name, ticket.job))
        out = np.empty(n, dtype=np.int32 if name in _INT_RESULTS else np.float64)
        if n and self._L.madam_b200_serve_result_copy(self._h, ticket.job, name.encode(),
                                                      out.ctypes.data_as(ct.c_void_p),
                                                      out.nbytes):
            raise RuntimeError("result copy failed")
        return out

    def info(self, ticket):
        """submit / start / end times (s), samples, PCG iterations, admitted
        bytes, and the setup / PCG / finalisation wall times (ms)."""
        out = np.zeros(9)
        if self._L.madam_b200_serve_job_info(self._h, ticket.job,
                                             out.ctypes.data_as(ct.c_void_p), 9):
            raise RuntimeError("job {} is not finished".format(ticket.job))
        keys = ("t_submit", "t_start", "t_end", "samples", "iterations", "bytes", "setup_ms",
                "iterate_ms", "finalize_ms")
        return dict(zip(keys, out.tolist()))

    def stats(self):
        """PCG rounds run by the stepper, job-rounds (jobs summed over the
        rounds) and the most jobs in one round."""
        out = np.zeros(3)
        self._L.madam_b200_serve_stats(self._h, out.ctypes.data_as(ct.c_void_p), 3)
        return dict(rounds=int(out[0]), job_rounds=int(out[1]), max_jobs=int(out[2]))

    def release(self, ticket):
        self._L.madam_b200_serve_release(self._h, ticket.job)
        ticket._keep = None

    def close(self):
        if self._h:
            self._L.madam_b200_serve_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
