"""Loader of the in-tree CUDA library libmadam.so (no CPU fallback).

The shared library exports the reference's C-ABI (destripe,
destripe_with_cache, clear_caches; madam.h:1-2, smadam.F90:593-951) plus
madam_b200_* entry points for status, results and benchmarking.
"""
import ctypes as ct
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmadam.so")

_lib = None


def build(force=False):
    """Compile libmadam.so for sm_100a with nvcc (in-tree)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-s", "-C", HERE, "-j4"], check=True)
    return LIB_PATH


def load():
    """Load libmadam.so; raises if the CUDA build is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("libmadam.so is not built: run libmadam_b200._lib.build() "
                           "(make -C libmadam_b200)")
    L = ct.CDLL(LIB_PATH)
    P = ct.c_void_p
    L.destripe.restype = None
    L.destripe_with_cache.restype = None
    L.clear_caches.restype = None
    L.clear_caches.argtypes = []
    L.madam_b200_destripe.restype = ct.c_int
    L.madam_b200_destripe.argtypes = [ct.c_int, ct.c_char_p, ct.c_long, ct.c_char_p, P, ct.c_long,
                                      ct.c_long, P, P, P, P, ct.c_long, P, P, ct.c_long, P,
                                      ct.c_long, P, ct.c_long, P]
    L.madam_b200_destripe_fp32.restype = ct.c_int
    L.madam_b200_destripe_fp32.argtypes = L.madam_b200_destripe.argtypes
    L.madam_b200_destripe_with_cache.restype = ct.c_int
    L.madam_b200_destripe_with_cache.argtypes = [ct.c_int, ct.c_long, ct.c_long, ct.c_long, P, P,
                                                 P, P, ct.c_char_p]
    L.madam_b200_destripe_with_cache_batch.restype = ct.c_int
    L.madam_b200_destripe_with_cache_batch.argtypes = [ct.c_int, ct.c_long, ct.c_long, ct.c_long,
                                                       P, P, P, ct.c_long, P]
    L.madam_b200_destripe_with_cache_batch_fp32.restype = ct.c_int
    L.madam_b200_destripe_with_cache_batch_fp32.argtypes = \
        L.madam_b200_destripe_with_cache_batch.argtypes
    L.madam_b200_clear_caches.restype = ct.c_int
    L.madam_b200_last_error.restype = ct.c_int
    L.madam_b200_last_error.argtypes = [ct.c_char_p, ct.c_long]
    L.madam_b200_result_size.restype = ct.c_long
    L.madam_b200_result_size.argtypes = [ct.c_char_p]
    L.madam_b200_result_copy.restype = ct.c_int
    L.madam_b200_result_copy.argtypes = [ct.c_char_p, P, ct.c_long]
    L.madam_b200_bench_iterations.restype = ct.c_int
    L.madam_b200_bench_iterations.argtypes = [ct.c_int, ct.c_int, P, ct.c_long]
    L.madam_b200_kernel_launches.restype = ct.c_ulonglong
    L.madam_b200_selftest_fastdiv.restype = ct.c_int
    _lib = L
    return L


def last_error():
    buf = ct.create_string_buffer(4096)
    status = load().madam_b200_last_error(buf, len(buf))
    return status, buf.value.decode(errors="replace")
