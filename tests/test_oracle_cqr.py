"""The oracle's complex QR restatement pinned without a GPU:

  * R and tau against LAPACK cgeqrf (same clarfg convention: beta = -sign(Re alpha) ||(alpha; x)||,
    real) and the reference's three Cgeqrf criteria (test/cgeqrf/data/verify_result.py:
    DQRT01 against f32 LAPACK's own ratio, A = Q R, Q^H Q = I) on the shapes of
    test/cgeqrf/test_cgeqrf.py:24;
  * Cungqr against LAPACK cungqr, Cunmqr (both sides, N and C) against an explicit Q and CCgels
    against lstsq, each within the operator tests' rtol 2e-4 / atol 3e-5
    (test/cungqr/test_cungqr.py:39, test/cunmqr/test_cunmqr.py:45, test/ccgels/test_ccgels.py:48),
    on their shapes;
  * CCgels' directed and singular cases (test/ccgels/test_ccgels.py:148-182);
  * the host argument ladders of the complex QR entries that reject before any device work."""

import ctypes as C

import numpy as np
import pytest

import oracle
from oracle import judges


def crand(m, n, seed):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n))).astype(np.complex64)


@pytest.mark.parametrize("m,n", [(1, 1), (7, 3), (3, 7), (65, 33), (257, 131), (40, 40), (100, 64), (33, 100),
                                 (1000, 40), (801, 64)])  # the last two: panels reduced in row segments
def test_cgeqrf_matches_lapack_and_passes_the_reference_criteria(m, n):
    from scipy.linalg import lapack

    a = crand(m, n, m * 17 + n)
    qr, tau = oracle.cgeqrf(a)
    lq, ltau, _, info = lapack.cgeqrf(np.asfortranarray(a.copy()))
    assert info == 0
    k = min(m, n)
    scale = np.abs(lq).max()
    assert np.abs(np.triu(qr[:k]) - np.triu(lq[:k])).max() <= 2e-5 * scale
    assert np.abs(tau - ltau[:k]).max() <= 2e-5
    ok, ratio, cpu = judges.cgeqrf_gate(a, qr, tau)
    assert ok, (ratio, cpu)


def test_cgeqrf_zero_column_and_real_alpha_give_tau_zero():
    a = crand(20, 6, 3)
    a[:, 2] = 0.0
    a[5:, 4] = 0.0
    qr, tau = oracle.cgeqrf(a)
    assert tau[2] == 0
    ok, _, _ = judges.cgeqrf_gate(a, qr, tau)
    assert ok
    # a column already upper triangular with a real diagonal needs no reflection
    b = np.zeros((5, 1), np.complex64)
    b[0, 0] = 3.0
    qr, tau = oracle.cgeqrf(b)
    assert tau[0] == 0 and qr[0, 0] == 3.0


@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (7, 5, 3), (65, 33, 17), (257, 131, 129), (7, 5, 0)])
def test_cungqr_matches_lapack(m, n, k):
    from scipy.linalg import lapack

    qr, tau = oracle.cgeqrf(crand(m, max(k, 1), m + n + k))
    tau = tau[:k]
    src = np.zeros((m, n), np.complex64)
    src[:, :k] = qr[:, :k]
    got = oracle.cungqr(src, tau, n)
    if k:
        want, _, info = lapack.cungqr(np.asfortranarray(src), tau)
        assert info == 0
    else:
        want = np.eye(m, n, dtype=np.complex64)
    assert judges.close_2e4(got, want)


@pytest.mark.parametrize("order,columns,k", [(7, 5, 3), (65, 33, 17), (257, 131, 129)])
def test_cunmqr_against_an_explicit_q(order, columns, k):
    qr, tau = oracle.cgeqrf(crand(order, order, order))
    tau = tau[:k]
    q = judges.cq_from_reflectors(qr, tau)
    for side in (0, 1):
        for herm in (0, 1):
            m, n = (order, columns) if side == 0 else (columns, order)
            c = crand(m, n, side * 2 + herm)
            got = oracle.cunmqr(side, herm, qr[:, :k], tau, c)
            op = q.conj().T if herm else q
            want = op @ c if side == 0 else c @ op
            assert judges.close_2e4(got, want), (side, herm)


@pytest.mark.parametrize("m,n,nrhs", [(7, 3, 1), (16, 16, 8), (65, 33, 3), (257, 131, 8)])
def test_cgels_matches_lstsq(m, n, nrhs):
    a, b = crand(m, n, m + n), crand(m, nrhs, nrhs)
    x, _, _, info = oracle.cgels(a, b)
    ref = np.linalg.lstsq(a.astype(np.complex128), b.astype(np.complex128), rcond=None)[0]
    assert info == 0 and judges.close_2e4(x, ref)


def test_cgels_directed_and_singular_cases():
    n = 16
    for j in (1, n - 1):
        b = np.zeros((n, 1), np.complex64)
        b[j, 0] = 1
        x, _, _, info = oracle.cgels(np.eye(n, dtype=np.complex64), b)
        assert info == 0 and np.array_equal(x, b)
    a = np.array([[1, 2], [3, 4]], np.complex64)
    x, _, _, info = oracle.cgels(a, np.array([[5], [6]], np.complex64))
    assert info == 0 and np.allclose(x[:, 0], [-4, 4.5], rtol=1e-5, atol=1e-6)
    a = np.zeros((3, 2), np.complex64)
    a[:, 0] = [1, 2, 3]
    x, _, _, info = oracle.cgels(a, np.ones((3, 1), np.complex64))
    assert info == 2 and np.all(x == 0)


def test_host_argument_ladders_without_a_gpu():
    import aclsolver

    lib = aclsolver.library()
    INVALID, NULL_HANDLE = 3, 9
    fake = C.c_void_p(16)  # never dereferenced by a query or an argument rejection
    lw = C.c_int(-1)
    assert lib.aclsolverCgeqrf_bufferSize(None, 4, 4, None, 4, C.byref(lw)) == NULL_HANDLE
    assert lib.aclsolverCgeqrf_bufferSize(fake, 10, 4, C.c_void_p(64), 10, C.byref(lw)) == 0 and lw.value == 2048
    assert lib.aclsolverCgeqrf_bufferSize(fake, 0, 4, None, 1, C.byref(lw)) == 0 and lw.value == 0
    assert lib.aclsolverCgeqrf_bufferSize(fake, 10, 4, None, 10, C.byref(lw)) == INVALID  # A null
    assert lib.aclsolverCgeqrf_bufferSize(fake, 10, 4, C.c_void_p(64), 9, C.byref(lw)) == INVALID
    assert lib.aclsolverCungqr_bufferSize(fake, 10, 6, 4, C.c_void_p(64), 10, C.c_void_p(64),
                                          C.byref(lw)) == 0 and lw.value == 1064
    assert lib.aclsolverCungqr_bufferSize(fake, 10, 11, 4, C.c_void_p(64), 10, C.c_void_p(64), C.byref(lw)) == INVALID
    assert lib.aclsolverCungqr_bufferSize(fake, 10, 6, 4, C.c_void_p(64), 10, None, C.byref(lw)) == INVALID
    p = C.c_void_p(64)
    assert lib.aclsolverCunmqr_bufferSize(fake, 0, 2, 10, 3, 4, p, 10, p, p, 10, C.byref(lw)) == 0 and lw.value == 1024
    assert lib.aclsolverCunmqr_bufferSize(fake, 0, 1, 10, 3, 4, p, 10, p, p, 10, C.byref(lw)) == INVALID  # OP_T
    assert lib.aclsolverCunmqr_bufferSize(fake, 1, 0, 10, 3, 4, p, 2, p, p, 10, C.byref(lw)) == INVALID  # lda < n
    assert lib.aclsolverCunmqr_bufferSize(fake, 0, 0, 10, 3, 0, None, 10, None, None, 10,
                                          C.byref(lw)) == 0 and lw.value == 0
    sz = C.c_size_t(1)
    assert lib.aclsolverCCgels_bufferSize(None, 10, 4, 1, p, 10, p, 10, p, 4, None, C.byref(sz)) == NULL_HANDLE
    assert lib.aclsolverCCgels_bufferSize(fake, 16, 16, 129, C.c_void_p(1 << 20), 16, C.c_void_p(2 << 20), 16,
                                          C.c_void_p(3 << 20), 16, None, C.byref(sz)) == INVALID
    assert lib.aclsolverCCgels_bufferSize(fake, 3, 4, 1, p, 3, p, 3, p, 4, None, C.byref(sz)) == INVALID  # m < n
    assert lib.aclsolverCCgels_bufferSize(fake, 0, 0, 0, None, 1, None, 1, None, 1, None, C.byref(sz)) == 0
    assert sz.value == 0
    info = C.c_int(5)
    # a null info: INVALID_VALUE, nothing written; a host info: not written either
    assert lib.aclsolverCgeqrf(fake, 4, 4, p, 4, p, p, 1024, None) == INVALID
    assert lib.aclsolverCgeqrf(fake, -1, 4, p, 4, p, p, 1024, C.byref(info)) == INVALID and info.value == 5
    assert lib.aclsolverCgeqrf(None, 4, 4, p, 4, p, p, 1024, C.byref(info)) == NULL_HANDLE
    niter = C.c_int(7)
    assert lib.aclsolverCCgels(fake, 4, 4, 1, p, 4, p, 4, p, 4, p, 1 << 20, None, C.byref(info)) == INVALID
    assert lib.aclsolverCCgels(fake, 4, 4, 1, p, 4, p, 4, p, 4, p, 1 << 20, C.byref(niter), None) == INVALID
