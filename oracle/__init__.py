"""The oracle: a CPU restatement of the reference's factor-and-solve arithmetic.

TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline may import this package; the library never does.  The arithmetic lives in
oracle.c (each routine cites the reference kernel it restates); this module is the numpy
front end over liboracle.so, plus the residual judges in judges.py.

All matrices here are numpy float32 arrays in column-major (Fortran) order, with shape
(count, n, n) for batches; views are made contiguous before the call.
"""

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIBRARY = HERE / "liboracle.so"

_F = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_I = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_VP = C.c_void_p
_i = C.c_int
_l = C.c_int64

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIBRARY.exists():
            raise RuntimeError(f"{LIBRARY} is missing: build it with `make -C oracle`")
        _lib = C.CDLL(str(LIBRARY))
        _lib.orc_spotrf_batched.argtypes = [_i, _F, _i, _l, _i, _i, _I, _i]
        _lib.orc_spotrs_batched.argtypes = [_i, _i, _F, _i, _l, _F, _i, _l, _i, _i, _i, _i]
        _lib.orc_sgetrf_batched.argtypes = [_i, _i, _F, _i, _l, _i, _VP, _I, _i]
        _lib.orc_sgetrs_batched.argtypes = [_i, _i, _i, _F, _i, _l, _VP, _F, _i, _l, _i, _i]
        _lib.orc_sgetri_batched.argtypes = [_i, _F, _i, _l, _VP, _F, _i, _l, _i, _I, _i]
        _lib.orc_cpotrf_batched.argtypes = [_i, _F, _i, _l, _i, _i, _I, _i]
        _lib.orc_cpotrs_batched.argtypes = [_i, _i, _F, _i, _l, _F, _i, _l, _i, _i, _i]
        _lib.orc_cgetrf_batched.argtypes = [_i, _i, _F, _i, _l, _i, _i, _I, _I, _i]
        _lib.orc_cgetri_batched.argtypes = [_i, _F, _i, _l, _VP, _F, _i, _l, _i, _I, _i]
        _lib.orc_cmatinv_batched.argtypes = [_i, _F, _i, _l, _F, _i, _l, _i, _I, _i]
        _lib.orc_cgetrs_batched.argtypes = [_i, _i, _i, _F, _i, _l, _VP, _F, _i, _l, _i, _i]
        _lib.orc_cdivide_many.argtypes = [_F, _F, _F, _l]
        _lib.orc_max_threads.restype = _i
    return _lib


def max_threads():
    return lib().orc_max_threads()


def _slab(a):
    """(count, n, m) column-major matrices -> contiguous float32 slab laid out as
    matrix q column j at offset q*m*n + j*n (i.e. the transpose in C order)."""
    a = np.asarray(a, dtype=np.float32)
    return np.array(a.transpose(0, 2, 1), dtype=np.float32, order="C", copy=True)


def _unslab(s):
    return np.ascontiguousarray(s.transpose(0, 2, 1))


def spotrf_batched(a, upper=False, threads=0):
    """In-place Cholesky of each (n, n) matrix; returns (factors, info)."""
    s = _slab(a)
    count, n = s.shape[0], s.shape[1]
    info = np.zeros(count, dtype=np.int32)
    lib().orc_spotrf_batched(n, s, n, n * n, count, int(upper), info, threads)
    return _unslab(s), info


def spotrs_batched(factors, b, upper=False, single=False, threads=0):
    """Solve L L^T x = b for (count, n, nrhs) right-hand sides in the order of
    SpotrsBatched, or of the single-matrix Spotrs when `single`."""
    fs = _slab(factors)
    bs = _slab(b)
    count, n = fs.shape[0], fs.shape[1]
    nrhs = bs.shape[1]
    lib().orc_spotrs_batched(n, nrhs, fs, n, n * n, bs, n, n * nrhs, count, int(upper), int(single), threads)
    return _unslab(bs)


def sgetrf_batched(a, pivoting=True, threads=0):
    """LU of each (m, n) matrix; returns (lu, ipiv (count, min(m,n)) 1-based, info)."""
    a = np.asarray(a, dtype=np.float32)
    count, m, n = a.shape
    s = np.array(a.transpose(0, 2, 1), dtype=np.float32, order="C", copy=True)  # column-major, lda = m
    steps = min(m, n)
    ipiv = np.zeros((count, steps), dtype=np.int32)
    info = np.zeros(count, dtype=np.int32)
    lib().orc_sgetrf_batched(m, n, s, m, m * n, count, ipiv.ctypes.data if pivoting else None, info, threads)
    return np.ascontiguousarray(s.transpose(0, 2, 1)), ipiv, info


def sgetrs_batched(lu, ipiv, b, trans=0, threads=0):
    """Solve op(A) x = b from LU factors; b (count, n, nrhs)."""
    ls = _slab(lu)
    bs = _slab(b)
    count, n = ls.shape[0], ls.shape[1]
    nrhs = bs.shape[1]
    piv = None if ipiv is None else np.ascontiguousarray(ipiv, dtype=np.int32)
    lib().orc_sgetrs_batched(
        int(trans), n, nrhs, ls, n, n * n, None if piv is None else piv.ctypes.data, bs, n, n * nrhs, count, threads
    )
    return _unslab(bs)


def sgetri_batched(lu, ipiv, threads=0):
    """Inverse from LU factors (vector-inverse order); returns (inverse, info)."""
    ls = _slab(lu)
    count, n = ls.shape[0], ls.shape[1]
    piv = None if ipiv is None else np.ascontiguousarray(ipiv, dtype=np.int32)
    out = np.zeros_like(ls)
    info = np.zeros(count, dtype=np.int32)
    lib().orc_sgetri_batched(
        n, ls, n, n * n, None if piv is None else piv.ctypes.data, out, n, n * n, count, info, threads
    )
    return _unslab(out), info


def _cslab(a):
    """(count, n, m) complex64 column-major matrices -> interleaved float32 slab."""
    a = np.asarray(a, dtype=np.complex64)
    t = np.array(a.transpose(0, 2, 1), dtype=np.complex64, order="C", copy=True)
    return t.view(np.float32).reshape(-1).copy(), t.shape


def _uncslab(flat, shape):
    return np.ascontiguousarray(flat.view(np.complex64).reshape(shape).transpose(0, 2, 1))


def cpotrf_batched(a, upper=False, threads=0):
    """In-place complex Cholesky of each (n, n) matrix; returns (factors, info)."""
    flat, shape = _cslab(a)
    count, n = shape[0], shape[1]
    info = np.zeros(count, dtype=np.int32)
    lib().orc_cpotrf_batched(n, flat, n, n * n, count, int(upper), info, threads)
    return _uncslab(flat, shape), info


def cpotrs_batched(factors, b, upper=False, threads=0):
    """Solve with complex Cholesky factors; b (count, n, nrhs)."""
    fa, fshape = _cslab(factors)
    fb, bshape = _cslab(b)
    count, n, nrhs = fshape[0], fshape[1], bshape[1]
    lib().orc_cpotrs_batched(n, nrhs, fa, n, n * n, fb, n, n * nrhs, count, int(upper), threads)
    return _uncslab(fb, bshape)


def cgetrf_batched(a, pivoting=True, threads=0):
    """Complex LU of each (m, n) matrix; returns (lu, ipiv (count, min(m, n)) 1-based, info)."""
    flat, shape = _cslab(a)
    count, n, m = shape
    steps = min(m, n)
    ipiv = np.zeros((count, max(steps, 1)), dtype=np.int32)
    info = np.zeros(count, dtype=np.int32)
    lib().orc_cgetrf_batched(m, n, flat, m, m * n, count, int(pivoting), ipiv, info, threads)
    return _uncslab(flat, shape), ipiv[:, :steps], info


def cgetri_batched(lu, ipiv, threads=0):
    """Inverse from complex LU factors (compensated column solves); returns (inverse, info).
    A matrix whose info is nonzero keeps a zero output here (the library leaves it unwritten)."""
    flat, shape = _cslab(lu)
    count, n = shape[0], shape[1]
    piv = None if ipiv is None else np.ascontiguousarray(ipiv, dtype=np.int32)
    out = np.zeros_like(flat)
    info = np.zeros(count, dtype=np.int32)
    lib().orc_cgetri_batched(n, flat, n, n * n, None if piv is None else piv.ctypes.data, out, n, n * n, count,
                             info, threads)
    return _uncslab(out, shape), info


def cmatinv_batched(a, threads=0):
    """Gauss-Jordan inverse of each (n, n) matrix; returns (inverse, info)."""
    flat, shape = _cslab(a)
    count, n = shape[0], shape[1]
    out = np.zeros_like(flat)
    info = np.zeros(count, dtype=np.int32)
    lib().orc_cmatinv_batched(n, flat, n, n * n, out, n, n * n, count, info, threads)
    return _uncslab(out, shape), info


def cgetrs_batched(lu, ipiv, b, trans=0, threads=0):
    """Solve op(A) x = b from complex LU factors; b (count, n, nrhs)."""
    fa, fshape = _cslab(lu)
    fb, bshape = _cslab(b)
    count, n, nrhs = fshape[0], fshape[1], bshape[1]
    piv = None if ipiv is None else np.ascontiguousarray(ipiv, dtype=np.int32)
    lib().orc_cgetrs_batched(int(trans), n, nrhs, fa, n, n * n, None if piv is None else piv.ctypes.data, fb, n,
                             n * nrhs, count, threads)
    return _uncslab(fb, bshape)


def cdivide(a, b):
    """Elementwise complex64 a / b in the reference's compensated division."""
    a = np.ascontiguousarray(a, dtype=np.complex64).reshape(-1)
    b = np.ascontiguousarray(b, dtype=np.complex64).reshape(-1)
    out = np.zeros_like(a)
    lib().orc_cdivide_many(a.view(np.float32), b.view(np.float32), out.view(np.float32), a.size)
    return out
