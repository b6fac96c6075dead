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
        _lib.orc_sgeqrf.argtypes = [_i, _i, _F, _i, _F]
        _lib.orc_sgeqr2_golden.argtypes = [_i, _i, _F, _i, _F]
        _lib.orc_sormqr.argtypes = [_i, _i, _i, _i, _i, _F, _i, _F, _F, _i]
        _lib.orc_sorgqr.argtypes = [_i, _i, _i, _F, _i, _F]
        _lib.orc_sgels.argtypes = [_i, _i, _i, _F, _i, _F, _i, _F, _i, _F]
        _lib.orc_slarft.argtypes = [_i, _i, _i, _F, _i, _F, _F, _i]
        _lib.orc_cgeqrf.argtypes = [_i, _i, _F, _i, _F]
        _lib.orc_cunmqr.argtypes = [_i, _i, _i, _i, _i, _F, _i, _F, _F, _i]
        _lib.orc_cungqr.argtypes = [_i, _i, _i, _F, _i, _F]
        _lib.orc_cgels.argtypes = [_i, _i, _i, _F, _i, _F, _i, _F, _i, _F]
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


def _cm(a):
    """2-D column-major float32 copy (as a flat C-contiguous array of the transpose)."""
    a = np.asarray(a, dtype=np.float32)
    return np.array(a.T, dtype=np.float32, order="C", copy=True).reshape(-1)


def _uncm(flat, rows, cols):
    return np.ascontiguousarray(flat.reshape(cols, rows).T)


def sgeqrf(a):
    """Blocked Householder QR of one (m, n) matrix; returns (R and V packed, tau)."""
    m, n = a.shape
    f = _cm(a)
    tau = np.zeros(max(1, min(m, n)), dtype=np.float32)
    lib().orc_sgeqrf(m, n, f, max(1, m), tau)
    return _uncm(f, m, n), tau[: min(m, n)]


def sgeqr2_golden(a):
    """The reference's unblocked CPU golden QR (sequential sums)."""
    m, n = a.shape
    f = _cm(a)
    tau = np.zeros(max(1, min(m, n)), dtype=np.float32)
    lib().orc_sgeqr2_golden(m, n, f, max(1, m), tau)
    return _uncm(f, m, n), tau[: min(m, n)]


def sormqr(side, trans, qr, tau, c):
    """op(Q) C (side 0) or C op(Q) (side 1) from packed reflectors; trans 0 = Q."""
    m, n = c.shape
    nq = qr.shape[0]
    k = len(tau)
    fa = _cm(qr)
    fc = _cm(c)
    t = np.ascontiguousarray(tau, dtype=np.float32)
    if t.size == 0:
        t = np.zeros(1, dtype=np.float32)
    lib().orc_sormqr(int(side), int(trans), m, n, k, fa, max(1, nq), t, fc, max(1, m))
    return _uncm(fc, m, n)


def sorgqr(qr, tau, n):
    """The first n columns of Q from packed reflectors (k = len(tau))."""
    m = qr.shape[0]
    k = len(tau)
    f = _cm(qr[:, :n] if qr.shape[1] >= n else np.pad(qr, ((0, 0), (0, n - qr.shape[1]))))
    t = np.ascontiguousarray(tau, dtype=np.float32)
    if t.size == 0:
        t = np.zeros(1, dtype=np.float32)
    lib().orc_sorgqr(m, n, k, f, max(1, m), t)
    return _uncm(f, m, n)


def sgels(a, b):
    """Least squares min ||A X - B|| (m >= n); returns (X, packed QR, tau)."""
    m, n = a.shape
    nrhs = b.shape[1]
    fa = _cm(a)
    fb = _cm(b)
    x = np.zeros(max(1, n) * max(1, nrhs), dtype=np.float32)
    tau = np.zeros(max(1, n), dtype=np.float32)
    lib().orc_sgels(m, n, nrhs, fa, max(1, m), fb, max(1, m), x, max(1, n), tau)
    return _uncm(x, max(1, n), max(1, nrhs))[:n, :nrhs], _uncm(fa, m, n), tau[:n]


def slarft(direct, v, tau, t_init=None):
    """T (k x k) of the block reflector of V (n x k) and tau; direct 0 forward, 1 backward.
    Entries outside the referenced triangle keep t_init (zeros by default)."""
    n, k = v.shape
    fv = _cm(v)
    t = _cm(np.zeros((k, k), np.float32) if t_init is None else t_init)
    tt = np.ascontiguousarray(tau, dtype=np.float32)
    lib().orc_slarft(int(direct), n, k, fv, max(1, n), tt if tt.size else np.zeros(1, np.float32), t, max(1, k))
    return _uncm(t, k, k)


def _ccm(a):
    """2-D complex64 column-major, as a flat float32 array."""
    a = np.asarray(a, dtype=np.complex64)
    return np.array(a.T, dtype=np.complex64, order="C", copy=True).reshape(-1).view(np.float32).copy()


def _unccm(flat, rows, cols):
    return np.ascontiguousarray(flat.view(np.complex64).reshape(cols, rows).T)


def _ctau(tau):
    t = np.ascontiguousarray(tau, dtype=np.complex64)
    return (t if t.size else np.zeros(1, np.complex64)).view(np.float32).copy()


def cgeqrf(a):
    """Complex Householder QR of one (m, n) matrix; returns (R and V packed, tau)."""
    m, n = a.shape
    f = _ccm(a)
    tau = np.zeros(2 * max(1, min(m, n)), dtype=np.float32)
    lib().orc_cgeqrf(m, n, f, max(1, m), tau)
    return _unccm(f, m, n), tau.view(np.complex64)[: min(m, n)].copy()


def cunmqr(side, herm, qr, tau, c):
    """op(Q) C (side 0) or C op(Q) (side 1); herm 1 applies Q^H."""
    m, n = c.shape
    nq = qr.shape[0]
    fc = _ccm(c)
    lib().orc_cunmqr(int(side), int(herm), m, n, len(tau), _ccm(qr), max(1, nq), _ctau(tau), fc, max(1, m))
    return _unccm(fc, m, n)


def cungqr(qr, tau, n):
    """The first n columns of Q (k = len(tau) reflectors in the leading columns of qr)."""
    m = qr.shape[0]
    src = np.zeros((m, n), dtype=np.complex64)
    kk = min(qr.shape[1], n)
    src[:, :kk] = qr[:, :kk]
    f = _ccm(src)
    lib().orc_cungqr(m, n, len(tau), f, max(1, m), _ctau(tau))
    return _unccm(f, m, n)


def cgels(a, b):
    """Complex least squares (m >= n); returns (X, packed QR, tau, info), info the one-based
    position of the first zero diagonal entry of R (X then zero) or 0."""
    m, n = a.shape
    nrhs = b.shape[1]
    fa = _ccm(a)
    x = np.zeros(2 * max(1, n) * max(1, nrhs), dtype=np.float32)
    tau = np.zeros(2 * max(1, n), dtype=np.float32)
    info = lib().orc_cgels(m, n, nrhs, fa, max(1, m), _ccm(b), max(1, m), x, max(1, n), tau)
    return (_unccm(x, max(1, n), max(1, nrhs))[:n, :nrhs], _unccm(fa, m, n), tau.view(np.complex64)[:n].copy(),
            int(info))
