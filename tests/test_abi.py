"""The C-ABI boundary: symbols, loading, argument validation without a GPU."""
import ctypes as ct
import os
import re

import numpy as np
import pytest

import libmadam_b200
from libmadam_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = []
    for h in ("madam.h", "madam_b200.h"):
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"\b([a-z_0-9]+)\s*\(", src)
    # (a function-pointer parameter's return type is not a symbol)
    skip = ("if", "sizeof", "void", "int", "long", "double", "char", "float")
    return sorted(set(n for n in names if n not in skip))


def test_library_builds_and_loads():
    libmadam_b200.build()
    L = _lib.load()
    assert os.path.exists(_lib.LIB_PATH)
    assert L is not None


def test_every_declared_symbol_is_exported():
    L = _lib.load()
    names = _declared()
    assert {"destripe", "destripe_with_cache", "clear_caches"} <= set(names)
    for n in names:
        assert hasattr(L, n), n


def test_reference_symbols_have_c_linkage():
    # the reference exports unmangled names (bind(c), smadam.F90:68,611,921)
    out = os.popen("nm -D --defined-only " + _lib.LIB_PATH).read()
    for n in ("destripe", "destripe_with_cache", "clear_caches"):
        assert re.search(r"\bT {}\b".format(n), out), n


def test_fastdiv_selftest():
    assert _lib.load().madam_b200_selftest_fastdiv() == 0


def test_parameter_errors_are_reported_not_aborted():
    from libmadam_b200 import libmadam_wrapper as W
    d = np.zeros(4)
    with pytest.raises(RuntimeError, match="Unknown parameter: bogus_key"):
        W.destripe(None, {"bogus_key": 1}, ["a"], np.ones(1), np.zeros(4), np.zeros(4, np.int32),
                   np.ones(4, np.float32), np.zeros(4), np.array([0]), np.ones(1, np.int64),
                   np.zeros(1), np.array([1.0, 2.0]), np.ones(2))
    with pytest.raises(RuntimeError, match="Failed to parse nside_map from x"):
        W.destripe(None, {"nside_map": "x"}, ["a"], np.ones(1), np.zeros(4),
                   np.zeros(4, np.int32), np.ones(4, np.float32), np.zeros(4), np.array([0]),
                   np.ones(1, np.int64), np.zeros(1), np.array([1.0, 2.0]), np.ones(2))
    with pytest.raises(RuntimeError, match="temperature_only=T but pointing weights are polarized"):
        W.destripe(None, {"temperature_only": True}, ["a"], np.ones(1), np.zeros(4),
                   np.zeros(4, np.int32), np.ones(12, np.float32), np.zeros(4), np.array([0]),
                   np.ones(1, np.int64), np.zeros(1), np.array([1.0, 2.0]), np.ones(2))
    status, msg = _lib.last_error()
    assert status == 1 and "polarized" in msg
    # nnz = 2: the reference's general pixel matrix is undefined (float32
    # weights handed to the float64 dsyr, smadam_routines.f90:227)
    with pytest.raises(RuntimeError, match="only nnz = 1 or nnz = 3 is supported"):
        W.destripe(None, {}, ["a"], np.ones(1), np.zeros(4), np.zeros(4, np.int32),
                   np.ones(8, np.float32), np.zeros(4), np.array([0]), np.ones(1, np.int64),
                   np.zeros(1), np.array([1.0, 2.0]), np.ones(2))
    del d


def test_destripe_with_cache_without_cache_fails():
    from libmadam_b200 import libmadam_wrapper as W
    W.clear_caches()
    with pytest.raises(RuntimeError, match="empty caches"):
        W.destripe_with_cache(None, np.zeros(4), np.zeros(4, np.int32), np.ones(4, np.float32),
                              np.zeros(4), b"")
    # the batched Monte Carlo calls read the same caches
    for fn in (W.destripe_with_cache_batch, W.destripe_with_cache_batch_fp32):
        with pytest.raises(RuntimeError, match="empty caches"):
            fn(None, np.zeros(4), np.zeros(4, np.int32), np.ones(4, np.float32),
               np.zeros((2, 4)))
    # no run, no results
    with pytest.raises(KeyError):
        W.get_result("map")


def test_void_entry_points_do_not_abort():
    L = _lib.load()
    p = ct.c_void_p
    z = np.zeros(8)
    L.destripe.argtypes = [ct.c_int, ct.c_char_p, ct.c_long, ct.c_char_p, p, ct.c_long, ct.c_long,
                           p, p, p, p, ct.c_long, p, p, ct.c_long, p, ct.c_long, p, ct.c_long, p]
    ptr = z.ctypes.data_as(p)
    per = np.zeros(1, np.int64)
    L.destripe(0, b"nside_map = 3;", 1, b"d;", ptr, 4, 1, ptr, ptr, ptr, ptr, 1,
               per.ctypes.data_as(p), per.ctypes.data_as(p), 1, ptr, 1, ptr, 1, ptr)
    status, msg = _lib.last_error()
    assert status == 1 and msg


def test_no_cpu_fallback_without_gpu():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from libmadam_b200 import libmadam_wrapper as W
    from libmadam_b200 import synthetic as syn
    d = syn.to_numpy(syn.generate(syn.small_config(nsamp_obs=256, nobs=1)))
    with pytest.raises(RuntimeError, match="CUDA"):
        W.destripe(None, d["pars"], d["dets"], d["detweights"], d["timestamps"], d["pixels"],
                   d["pixweights"], d["signal"], d["periods"], d["npsd"], d["psdstarts"],
                   d["psdfreqs"], d["psdvals"])


class _FakeMpiComm:
    """Stands in for an mpi4py communicator (Get_size, py2f)."""

    def __init__(self, size, handle):
        self._size, self._handle = size, handle

    def Get_size(self):
        return self._size

    def py2f(self):
        return self._handle


def test_multi_rank_mpi_communicator_is_refused():
    # the reference reduces over its MPI communicator (smadam.F90:115-117);
    # this library does not, so N MPI ranks must not become N one-rank solves
    from libmadam_b200 import libmadam_wrapper as W
    with pytest.raises(ValueError, match="communicator of 2 ranks"):
        W._fcomm(_FakeMpiComm(2, 0))
    with pytest.raises(ValueError, match="communicator of 2 ranks"):
        W.destripe(_FakeMpiComm(2, 0), {}, ["a"], np.ones(1), np.zeros(4),
                   np.zeros(4, np.int32), np.ones(4, np.float32), np.zeros(4), np.array([0]),
                   np.ones(1, np.int64), np.zeros(1), np.array([1.0, 2.0]), np.ones(2))
    # one rank (MPI_COMM_SELF is Fortran handle 1 in Open MPI) runs one rank,
    # whatever its handle
    assert W._fcomm(_FakeMpiComm(1, 1)) == 0
    assert W._fcomm(None) == 0


def test_library_handles_avoid_mpi_fortran_handles():
    src = open(os.path.join(ROOT, "libmadam_b200", "csrc", "comm.cu")).read()
    first = int(re.search(r"kFirstHandle = (0x[0-9A-Fa-f]+)", src).group(1), 16)
    # Open MPI: small indices; MPICH built-ins 0x44000000.., created ones negative
    assert 1 << 16 < first < 0x44000000 - (1 << 20)


@pytest.mark.parametrize("case, msg", [
    ("nofile", "cannot open"),
    ("header", "is not formatted correctly"),
    ("missing", "ERROR: a not in"),
    ("short", "Failed to read the table from spectrum file"),
    ("slash", "Failed to read detector noise levels"),
    ("null", "Failed to read detector noise levels"),
])
def test_bad_spectrum_file_fails_before_device_work(tmp_path, case, msg):
    """A lone rank reads file_spectrum (read_spectrum,
    noise_routines.f90:505-596) before any device work: its errors need no
    GPU."""
    from libmadam_b200 import libmadam_wrapper as W
    path = tmp_path / "spec.txt"
    rows = ["%g %g" % (f, 1e-6 / f) for f in (0.01, 0.1, 1.0)]
    text = ["3 1", "b" if case == "missing" else "a_det", "1e-3"] + rows
    if case == "header":
        text[0] = "three one"
    elif case == "short":
        text = text[:-1]
    elif case == "slash":
        text[2] = "/ 1e-3"
    elif case == "null":
        text[2] = "1* 1e-3"
    if case != "nofile":
        path.write_text("\n".join(text) + "\n")
    with pytest.raises(RuntimeError, match=msg):
        W.destripe(None, {"kfilter": True, "file_spectrum": str(path)}, ["a"], np.ones(1),
                   np.zeros(4), np.zeros(4, np.int32), np.ones(4, np.float32), np.zeros(4),
                   np.array([0]), np.ones(1, np.int64), np.zeros(1), np.array([1.0, 2.0]),
                   np.ones(2))


def test_spectrum_file_with_repeat_counts_is_read():
    """Repeat counts ("r*c") and quoted names read as the reference's
    list-directed READ reads them: the call gets past the file (and then
    needs a GPU)."""
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import tempfile
    from libmadam_b200 import libmadam_wrapper as W
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "spec.txt")
        with open(path, "w") as f:
            f.write("3, 2  header words\n'x_a', \"b\"\n2*1d-3\n")
            for fr in (0.01, 0.1, 1.0):
                f.write("%g 2*%g\n" % (fr, 1e-6 / fr))
        with pytest.raises(RuntimeError, match="CUDA"):
            W.destripe(None, {"kfilter": True, "file_spectrum": path}, ["a"], np.ones(1),
                       np.zeros(4), np.zeros(4, np.int32), np.ones(4, np.float32), np.zeros(4),
                       np.array([0]), np.ones(1, np.int64), np.zeros(1), np.array([1.0, 2.0]),
                       np.ones(2))


def test_server_arguments_and_no_cpu_fallback():
    """The job server checks its arguments, and without a GPU it refuses to
    open rather than serving on the CPU."""
    from libmadam_b200.serve import Server
    with pytest.raises(RuntimeError, match="nworkers must be in 1..64"):
        Server(workers=0)
    with pytest.raises(RuntimeError, match=r"mem_fraction must be in \(0, 1\]"):
        Server(workers=2, mem_fraction=0.0)
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        return
    with pytest.raises(RuntimeError, match="CUDA"):
        Server(workers=2)
