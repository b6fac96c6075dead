"""The complex QR family on the GPU through the C ABI: Cgeqrf, Cunmqr (both sides, N and C),
Cungqr and CCgels, each bit for bit the oracle's blocked restatement (orc_cgeqrf / orc_cunmqr
/ orc_cungqr / orc_cgels), with the reference's acceptance criteria on top
(test/cgeqrf/data/verify_result.py; rtol 2e-4 / atol 3e-5 in test/cungqr/test_cungqr.py:39,
test/cunmqr/test_cunmqr.py:45, test/ccgels/test_ccgels.py:48), its padding checks, its
non-finite screening and its argument ladders."""

import ctypes as C

import numpy as np
import pytest
import torch

import aclsolver
import oracle
from oracle import judges
from helpers import info_buffer
from test_gpu_complex import CMatrices, cbits

pytestmark = pytest.mark.gpu

LEFT, RIGHT = 0, 1
OP_N, OP_T, OP_C = 0, 1, 2


def crand(m, n, seed):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n))).astype(np.complex64)


def cwork(elems):
    return torch.full((2 * max(1, elems),), float("nan"), dtype=torch.float32, device="cuda")


def ctensor(x):
    x = np.ascontiguousarray(x, dtype=np.complex64)
    return torch.from_numpy((x if x.size else np.zeros(1, np.complex64)).view(np.float32).copy()).cuda()


def geqrf(handle, a, pad=3):
    lib = aclsolver.library()
    m, n = a.shape
    dm = CMatrices(a[None], m + pad)
    tau = cwork(min(m, n))
    lw = C.c_int(-1)
    assert lib.aclsolverCgeqrf_bufferSize(handle.value, m, n, dm.tensor.data_ptr(), dm.ld,
                                          C.byref(lw)) == aclsolver.SUCCESS
    w = cwork(lw.value)
    info = info_buffer(1)
    st = lib.aclsolverCgeqrf(handle.value, m, n, dm.tensor.data_ptr(), dm.ld, tau.data_ptr(), w.data_ptr(), lw.value,
                             info.data_ptr())
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS and int(info.cpu()[0]) == 0
    return dm.read()[0], tau.cpu().numpy().view(np.complex64)[: min(m, n)]


@pytest.mark.parametrize("m,n", [(1, 1), (7, 3), (3, 7), (65, 33), (257, 131), (2, 2), (32, 32), (33, 33),
                                 (100, 64), (300, 257), (257, 300), (1000, 200), (4096, 40), (1024, 1024),
                                 (801, 64), (7000, 33)])
def test_cgeqrf_matches_oracle(handle, m, n):
    a = crand(m, n, m * 29 + n)
    got, tau = geqrf(handle, a)
    want, wtau = oracle.cgeqrf(a)
    assert cbits(tau, wtau)
    assert cbits(got, want)


def test_cgeqrf_passes_the_reference_criteria(handle):
    a = crand(1024, 256, 11)  # the reference's default verify_result.py shape
    got, tau = geqrf(handle, a)
    ok, ratio, cpu = judges.cgeqrf_gate(a, got, tau)
    assert ok, (ratio, cpu)


def test_cgeqrf_zero_columns(handle):
    a = crand(200, 150, 5)
    a[:, 7] = 0.0
    a[120:, 40] = 0.0
    a[41:, 41] = 0.0
    a[41, 41] = 2.5  # already reduced with a real diagonal: tau 0
    got, tau = geqrf(handle, a)
    want, wtau = oracle.cgeqrf(a)
    assert cbits(got, want) and cbits(tau, wtau)
    assert tau[7] == 0


def unmqr(handle, side, trans, qr, tau, c, pad=2):
    lib = aclsolver.library()
    m, n = c.shape
    k = len(tau)
    nq = qr.shape[0]
    da = CMatrices(qr[None], nq + 1)
    dc = CMatrices(c[None], m + pad)
    dt = ctensor(tau)
    lw = C.c_int(-1)
    assert lib.aclsolverCunmqr_bufferSize(handle.value, side, trans, m, n, k, da.tensor.data_ptr(), da.ld,
                                          dt.data_ptr(), dc.tensor.data_ptr(), dc.ld, C.byref(lw)) == aclsolver.SUCCESS
    w = cwork(lw.value)
    info = info_buffer(1)
    st = lib.aclsolverCunmqr(handle.value, side, trans, m, n, k, da.tensor.data_ptr(), da.ld, dt.data_ptr(),
                             dc.tensor.data_ptr(), dc.ld, w.data_ptr(), lw.value, info.data_ptr())
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS and int(info.cpu()[0]) == 0
    assert da.unchanged()
    return dc.read()[0]


@pytest.mark.parametrize("side", [LEFT, RIGHT])
@pytest.mark.parametrize("trans", [OP_N, OP_C])
@pytest.mark.parametrize("order,columns,k", [(7, 5, 3), (65, 33, 17), (257, 131, 129), (300, 40, 300)])
def test_cunmqr_matches_oracle_and_the_reference_tolerance(handle, side, trans, order, columns, k):
    qr, tau = oracle.cgeqrf(crand(order, order, order + k))
    qr, tau = qr[:, :k], tau[:k]
    m, n = (order, columns) if side == LEFT else (columns, order)
    c = crand(m, n, side * 3 + trans)
    got = unmqr(handle, side, trans, qr, tau, c)
    assert cbits(got, oracle.cunmqr(side, int(trans == OP_C), qr, tau, c))
    q = judges.cq_from_reflectors(qr, tau)
    op = q.conj().T if trans == OP_C else q
    assert judges.close_2e4(got, op @ c if side == LEFT else c @ op)


def ungqr(handle, src, tau, n):
    lib = aclsolver.library()
    m = src.shape[0]
    k = len(tau)
    dm = CMatrices(src[None], m + 8)
    dt = ctensor(tau)
    lw = C.c_int(-1)
    assert lib.aclsolverCungqr_bufferSize(handle.value, m, n, k, dm.tensor.data_ptr(), dm.ld, dt.data_ptr(),
                                          C.byref(lw)) == aclsolver.SUCCESS
    w = cwork(lw.value)
    info = info_buffer(1)
    st = lib.aclsolverCungqr(handle.value, m, n, k, dm.tensor.data_ptr(), dm.ld, dt.data_ptr(), w.data_ptr(),
                             lw.value, info.data_ptr())
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS and int(info.cpu()[0]) == 0
    return dm.read()[0]


@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (7, 5, 3), (65, 33, 17), (257, 131, 129), (7, 5, 0),
                                   (300, 300, 257), (1000, 100, 100)])
def test_cungqr_matches_oracle_and_lapack(handle, m, n, k):
    from scipy.linalg import lapack

    qr, tau = oracle.cgeqrf(crand(m, max(k, 1), m + n + k))
    tau = tau[:k]
    src = np.zeros((m, n), np.complex64)
    src[:, :k] = qr[:, :k]
    got = ungqr(handle, src, tau, n)
    assert cbits(got, oracle.cungqr(src, tau, n))
    want = lapack.cungqr(np.asfortranarray(src), tau)[0] if k else np.eye(m, n, dtype=np.complex64)
    assert judges.close_2e4(got, want)


def gels(handle, a, b, pad=8, expect=aclsolver.SUCCESS):
    lib = aclsolver.library()
    m, n = a.shape
    nrhs = b.shape[1]
    da = CMatrices(a[None], m + pad)
    db = CMatrices(b[None], m + pad)
    dx = CMatrices(np.zeros((1, n, nrhs), np.complex64), n + pad)
    sz = C.c_size_t(0)
    assert lib.aclsolverCCgels_bufferSize(handle.value, m, n, nrhs, da.tensor.data_ptr(), da.ld, db.tensor.data_ptr(),
                                          db.ld, dx.tensor.data_ptr(), dx.ld, None, C.byref(sz)) == aclsolver.SUCCESS
    w = torch.empty(max(1, sz.value), dtype=torch.uint8, device="cuda")
    info = info_buffer(1)
    niter = C.c_int(-5)
    st = lib.aclsolverCCgels(handle.value, m, n, nrhs, da.tensor.data_ptr(), da.ld, db.tensor.data_ptr(), db.ld,
                             dx.tensor.data_ptr(), dx.ld, w.data_ptr(), sz.value, C.byref(niter), info.data_ptr())
    handle.stream.synchronize()
    assert st == expect and niter.value == 0
    assert db.unchanged()
    return dx, int(info.cpu()[0])


@pytest.mark.parametrize("m,n,nrhs", [(7, 3, 1), (16, 16, 8), (65, 33, 3), (257, 131, 8), (1000, 500, 16),
                                      (1024, 1024, 4)])
def test_ccgels_matches_oracle_and_lstsq(handle, m, n, nrhs):
    a, b = crand(m, n, m + n), crand(m, nrhs, nrhs)
    dx, info = gels(handle, a, b)
    x = dx.read()[0]
    want, _, _, winfo = oracle.cgels(a, b)
    assert info == winfo == 0
    assert cbits(x, want)
    if m <= 1000:
        ref = np.linalg.lstsq(a.astype(np.complex128), b.astype(np.complex128), rcond=None)[0]
        assert judges.close_2e4(x, ref)


def test_ccgels_boundary_directed_and_singular(handle):
    """test/ccgels/test_ccgels.py:130-182: A = I at n = 4096, nrhs = 128 (x = b); e_j right-hand
    sides; a zero column (dinfo 2, X untouched)."""
    rng = np.random.default_rng(5321)
    b = (rng.normal(size=(4096, 128)) + 1j * rng.normal(size=(4096, 128))).astype(np.complex64)
    dx, info = gels(handle, np.eye(4096, dtype=np.complex64), b)
    assert info == 0 and np.allclose(dx.read()[0], b, rtol=1e-5, atol=1e-5)
    for j in (1, 15):
        e = np.zeros((16, 1), np.complex64)
        e[j, 0] = 1
        dx, info = gels(handle, np.eye(16, dtype=np.complex64), e)
        assert info == 0 and np.array_equal(dx.read()[0], e)
    a = np.zeros((3, 2), np.complex64)
    a[:, 0] = [1, 2, 3]
    dx, info = gels(handle, a, np.ones((3, 1), np.complex64))
    assert info == 2 and dx.unchanged()


def test_nonfinite_inputs_are_rejected_after_a_screen(handle):
    lib = aclsolver.library()
    a = crand(40, 20, 1)
    a[33, 5] = np.complex64(complex(0, np.inf))
    dm = CMatrices(a[None], 41)
    tau, w, info = cwork(20), cwork(2048), info_buffer(1)
    st = lib.aclsolverCgeqrf(handle.value, 40, 20, dm.tensor.data_ptr(), 41, tau.data_ptr(), w.data_ptr(), 2048,
                             info.data_ptr())
    handle.stream.synchronize()
    assert st == aclsolver.INVALID_VALUE and int(info.cpu()[0]) == -3 and dm.unchanged()
    # Cunmqr: a NaN above the diagonal of the reflector store is not an input; one in C is (-9)
    qr, t = oracle.cgeqrf(crand(30, 30, 2))
    qr[2, 10] = np.nan
    c = crand(30, 4, 3)
    got = unmqr(handle, LEFT, OP_N, qr[:, :12], t[:12], c)
    assert cbits(got, oracle.cunmqr(0, 0, qr[:, :12], t[:12], c))
    c[4, 2] = np.nan
    da, dc, dt = CMatrices(qr[None, :, :12], 30), CMatrices(c[None], 30), ctensor(t[:12])
    st = lib.aclsolverCunmqr(handle.value, LEFT, OP_N, 30, 4, 12, da.tensor.data_ptr(), 30, dt.data_ptr(),
                             dc.tensor.data_ptr(), 30, w.data_ptr(), 1024, info.data_ptr())
    handle.stream.synchronize()
    assert st == aclsolver.INVALID_VALUE and int(info.cpu()[0]) == -9 and dc.unchanged()
    # CCgels: A and B both non-finite -> the smaller index, -4
    a, b = crand(10, 10, 4), crand(10, 2, 5)
    a[0, 0], b[1, 1] = np.nan, np.inf
    dx, code = gels(handle, a, b, expect=aclsolver.INVALID_VALUE)
    assert code == -4 and dx.unchanged()


def test_argument_ladders_write_minus_the_index(handle):
    lib = aclsolver.library()
    a = crand(16, 16, 9)
    d = CMatrices(a[None], 16)
    p = d.tensor.data_ptr()
    tau, w = cwork(16), cwork(2048)
    info = info_buffer(1)

    def code():
        handle.stream.synchronize()
        return int(info.cpu()[0])

    assert lib.aclsolverCgeqrf(handle.value, 16, 16, p, 16, None, w.data_ptr(), 2048, info.data_ptr()) == 3
    assert code() == -5
    assert lib.aclsolverCgeqrf(handle.value, 16, 16, p, 16, tau.data_ptr(), w.data_ptr(), 2047, info.data_ptr()) == 3
    assert code() == -7
    assert lib.aclsolverCgeqrf(handle.value, 16, 16, p, 16, tau.data_ptr(), None, 2048, info.data_ptr()) == 3
    assert code() == -6
    assert lib.aclsolverCgeqrf(handle.value, 0, 16, None, 1, None, None, 0, info.data_ptr()) == 0 and code() == 0
    assert lib.aclsolverCungqr(handle.value, 16, 17, 4, p, 16, tau.data_ptr(), w.data_ptr(), 2048,
                               info.data_ptr()) == 3 and code() == -2
    assert lib.aclsolverCungqr(handle.value, 16, 8, 4, p, 16, tau.data_ptr(), w.data_ptr(), 64,
                               info.data_ptr()) == 3 and code() == -8
    assert lib.aclsolverCunmqr(handle.value, LEFT, OP_T, 16, 4, 4, p, 16, tau.data_ptr(), p, 16, w.data_ptr(), 1024,
                               info.data_ptr()) == 3 and code() == -2
    assert lib.aclsolverCunmqr(handle.value, RIGHT, OP_N, 4, 16, 4, p, 16, tau.data_ptr(), p, 3, w.data_ptr(), 1024,
                               info.data_ptr()) == 3 and code() == -10
    niter = C.c_int(0)
    big = cwork(16 * 130)  # dB and dX with room for 129 columns, so only the count is wrong
    xb = cwork(16 * 130)
    assert lib.aclsolverCCgels(handle.value, 16, 16, 129, p, 16, big.data_ptr(), 16, xb.data_ptr(), 16, w.data_ptr(),
                               1 << 20, C.byref(niter), info.data_ptr()) == 3 and code() == -3
    assert lib.aclsolverCCgels(handle.value, 16, 16, 1, p, 16, p, 16, p, 16, w.data_ptr(), 1 << 20, C.byref(niter),
                               info.data_ptr()) == 3 and code() == -8  # dX = dA
    assert lib.aclsolverCCgels(handle.value, 16, 16, 1, p, 16, big.data_ptr(), 16, xb.data_ptr(), 16, w.data_ptr(), 8,
                               C.byref(niter), info.data_ptr()) == 3 and code() == -11
    assert lib.aclsolverCCgels(handle.value, 16, 16, 1, p, 16, big.data_ptr(), 16, xb.data_ptr(), 16, w.data_ptr(),
                               1 << 20, None, info.data_ptr()) == 3 and code() == -12


def test_cgeqrf_look_ahead_on_a_side_stream():
    """On a non-default stream the look-ahead forks and joins its panel stream around the
    caller's work: the result is the oracle's bits and later work on the stream sees it."""
    lib = aclsolver.library()
    m, n = 900, 700
    a = crand(m, n, 123)
    stream = torch.cuda.Stream()
    with aclsolver.Handle(stream=stream) as h:
        dm = CMatrices(a[None], m + 2)
        tau = cwork(n)
        lw = C.c_int(-1)
        assert lib.aclsolverCgeqrf_bufferSize(h.value, m, n, dm.tensor.data_ptr(), dm.ld, C.byref(lw)) == 0
        w = cwork(lw.value)
        info = info_buffer(1)
        copy = torch.empty_like(dm.tensor)
        torch.cuda.synchronize()  # the buffers were filled on the default stream
        with torch.cuda.stream(stream):
            assert lib.aclsolverCgeqrf(h.value, m, n, dm.tensor.data_ptr(), dm.ld, tau.data_ptr(), w.data_ptr(),
                                       lw.value, info.data_ptr()) == aclsolver.SUCCESS
            copy.copy_(dm.tensor)  # ordered after the call on the same stream
        stream.synchronize()
        want, wtau = oracle.cgeqrf(a)
        got = np.ascontiguousarray(copy.cpu().numpy().view(np.complex64).reshape(n, m + 2)[:, :m].T)
        assert int(info.cpu()[0]) == 0
        assert cbits(got, want) and cbits(tau.cpu().numpy().view(np.complex64)[:n], wtau)


@pytest.mark.parametrize("m,n", [(4100, 70), (513, 200), (700, 1000), (801, 97), (6401, 40)])
def test_cgeqrf_shape_sweep(handle, m, n):
    """Shapes around the panel thresholds (one block up to 800 rows, an eight-block cluster up
    to 6,400, then one block reading A), and the look-ahead's, against the oracle."""
    a = crand(m, n, m + 3 * n)
    got, tau = geqrf(handle, a, pad=1)
    want, wtau = oracle.cgeqrf(a)
    assert cbits(tau, wtau) and cbits(got, want)
