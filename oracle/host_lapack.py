"""The host LAPACK the reference's tests use as their golden (scipy's bundled OpenBLAS),
driven over whole batches from C (lapack_host.c) for the benchmark's CPU baseline.

BENCHMARK AND TEST INFRASTRUCTURE ONLY: the library never imports this module.

The reference compares its device results with scipy's FP32 LAPACK
(test/cholesky/lapack_residual.py:64-86, test/utils/cholesky/fixtures.py:108-136).  scipy
ships OpenBLAS as scipy.libs/libscipy_openblas*.so with the LAPACKE interface exported under
a scipy_ prefix; liblapackhost.so opens that file and calls it with OpenMP over matrices
(one OpenBLAS thread per call) or, for one large system, with OpenBLAS's own threads.

All arrays are flat float32 buffers of column-major matrices laid end to end.
"""

import ctypes as C
import os
import platform
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIBRARY = HERE / "liblapackhost.so"

_F = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_I = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_L = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_i = C.c_int

_lib = None


def openblas_path():
    """scipy's bundled OpenBLAS (the library scipy.linalg.lapack calls)."""
    import scipy

    libs = Path(scipy.__file__).resolve().parent.parent / "scipy.libs"
    found = sorted(libs.glob("libscipy_openblas*.so"))
    if not found:
        raise RuntimeError(f"no libscipy_openblas*.so under {libs}")
    return found[0]


def lib():
    global _lib
    if _lib is None:
        if not LIBRARY.exists():
            raise RuntimeError(f"{LIBRARY} is missing: build it with `make -C oracle`")
        h = C.CDLL(str(LIBRARY))
        h.lh_open.argtypes = [C.c_char_p]
        h.lh_config.restype = C.c_char_p
        h.lh_potrf_potrs_batched.argtypes = [_i, _i, _i, _F, _F, _F, _F, _i, _I, _i]
        h.lh_getrf_getrs_batched.argtypes = [_i, _i, _F, _F, _F, _F, C.c_void_p, _I, _i, _I, _i]
        h.lh_cpotrf_cpotrs_vbatched.argtypes = [_I, _L, _L, _F, _F, _F, _F, _i, _i, _I, _i]
        h.lh_sgesv_single.argtypes = [_i, _i, _F, _F, _F, _F, _I, _i]
        h.lh_spotrf_single.argtypes = [_i, _F, _F, _i]
        if h.lh_open(str(openblas_path()).encode()) != 0:
            raise RuntimeError(f"could not load the LAPACKE symbols from {openblas_path()}")
        _lib = h
    return _lib


def describe(threads):
    """What the baseline ran on: CPU model, the host's logical CPUs, the threads used."""
    model = platform.processor() or "unknown"
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return {"cpu_model": model, "host_cpus": os.cpu_count(), "cores": threads,
            "library": f"OpenBLAS via scipy ({lib().lh_config().decode(errors='replace')})"}


def max_threads():
    return lib().lh_max_threads()


def potrf_potrs(n, nrhs, a, b, count, upper=False, threads=0):
    """spotrf + spotrs over `count` matrices; returns (factors, solutions, info)."""
    w, x = np.empty_like(a), np.empty_like(b)
    info = np.zeros(count, dtype=np.int32)
    lib().lh_potrf_potrs_batched(n, nrhs, int(upper), a, w, b, x, count, info, threads or max_threads())
    return w, x, info


def getrf_getrs(n, nrhs, a, b, count, inverse=False, threads=0):
    """sgetrf + sgetrs (+ sgetri of a copy of the factor); returns (lu, x, inv, ipiv, info)."""
    w, x = np.empty_like(a), np.empty_like(b)
    inv = np.empty_like(a) if inverse else None
    ipiv = np.zeros(count * n, dtype=np.int32)
    info = np.zeros(count, dtype=np.int32)
    lib().lh_getrf_getrs_batched(n, nrhs, a, w, b, x, None if inv is None else inv.ctypes.data, ipiv, count, info,
                                 threads or max_threads())
    return w, x, inv, ipiv, info


def cpotrf_cpotrs_vbatched(orders, a_off, b_off, a, b, nrhs, threads=0):
    """complex64 cpotrf + cpotrs over matrices of different orders (offsets in floats)."""
    w, x = np.empty_like(a), np.empty_like(b)
    orders = np.ascontiguousarray(orders, dtype=np.int32)
    info = np.zeros(len(orders), dtype=np.int32)
    lib().lh_cpotrf_cpotrs_vbatched(orders, np.ascontiguousarray(a_off, dtype=np.int64),
                                    np.ascontiguousarray(b_off, dtype=np.int64), a, w, b, x, nrhs, len(orders), info,
                                    threads or max_threads())
    return w, x, info


def sgesv(n, nrhs, a, b, threads=0):
    """One system: sgetrf + sgetrs with OpenBLAS threaded; returns (x, info)."""
    w, x = np.empty_like(a), np.empty_like(b)
    ipiv = np.zeros(n, dtype=np.int32)
    st = lib().lh_sgesv_single(n, nrhs, a, w, b, x, ipiv, threads or max_threads())
    return x, st


def spotrf(n, a, threads=0):
    """One matrix: spotrf (lower) with OpenBLAS threaded; returns (factor, info)."""
    w = np.empty_like(a)
    st = lib().lh_spotrf_single(n, a, w, threads or max_threads())
    return w, st
