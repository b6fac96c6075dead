"""The real QR family on the GPU through the C ABI: Sgeqrf, Sormqr (both sides, all
operations), Sorgqr and SSgels, each bit for bit the oracle's blocked restatement
(orc_sgeqrf / orc_sormqr / orc_sorgqr / orc_sgels), with the reference's acceptance gates
(test/sgeqrf/sgeqrf_test.cpp:16, test/sgels/sgels_test.cpp:16-24) on top."""

import ctypes as C

import numpy as np
import pytest
import torch

import aclsolver
import oracle
from oracle import judges
from helpers import DeviceMatrices, info_buffer, same_bits

pytestmark = pytest.mark.gpu

LEFT, RIGHT = 0, 1
OP_N, OP_T, OP_C = 0, 1, 2


def rand(m, n, seed):
    return np.random.default_rng(seed).standard_normal((m, n)).astype(np.float32)


def work(floats):
    return torch.full((max(1, floats),), float("nan"), dtype=torch.float32, device="cuda")


def geqrf(handle, a, pad=0):
    lib = aclsolver.library()
    m, n = a.shape
    dm = DeviceMatrices(a, m + pad)
    tau = torch.full((max(1, min(m, n)),), float("nan"), dtype=torch.float32, device="cuda")
    lw = C.c_int(-1)
    assert lib.aclsolverSgeqrf_bufferSize(handle.value, m, n, dm.ptr, dm.ld, C.byref(lw)) == aclsolver.SUCCESS
    w = work(lw.value)
    info = info_buffer(1)
    st = lib.aclsolverSgeqrf(handle.value, m, n, dm.ptr, dm.ld, tau.data_ptr(), w.data_ptr(), lw.value,
                             info.data_ptr())
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS and int(info.cpu()[0]) == 0
    return dm.read()[0], tau.cpu().numpy()[: min(m, n)]


@pytest.mark.parametrize("m,n", [(1, 1), (2, 2), (18, 8), (32, 4), (57, 57), (66, 8), (100, 33), (33, 100),
                                 (300, 257), (257, 300), (1000, 200), (4096, 64), (1024, 1024), (2500, 100),
                                 (1700, 33)])
def test_sgeqrf_matches_oracle(handle, m, n):
    a = rand(m, n, m * 13 + n)
    got, tau = geqrf(handle, a, pad=3)
    want, wtau = oracle.sgeqrf(a)
    assert same_bits(tau, wtau)
    assert same_bits(got, want)


def test_sgeqrf_zero_columns_and_the_reference_gate(handle):
    a = rand(200, 150, 5)
    a[:, 7] = 0.0
    a[120:, 40] = 0.0
    got, tau = geqrf(handle, a)
    want, wtau = oracle.sgeqrf(a)
    assert same_bits(got, want) and same_bits(tau, wtau)
    g, gtau = oracle.sgeqr2_golden(a)
    assert judges.qr_ratio(a, got, tau) <= max(5 * judges.qr_ratio(a, g, gtau), 0.1)


def sormqr(handle, side, trans, qr, tau, c, pad=2):
    lib = aclsolver.library()
    m, n = c.shape
    k = len(tau)
    nq = qr.shape[0]
    da = DeviceMatrices(qr, nq + 1)
    dc = DeviceMatrices(c, m + pad)
    dt = torch.tensor(np.ascontiguousarray(tau), device="cuda")
    lw = C.c_int(-1)
    assert lib.aclsolverSormqr_bufferSize(handle.value, side, trans, m, n, k, da.ptr, da.ld, dt.data_ptr(), dc.ptr,
                                          dc.ld, C.byref(lw)) == aclsolver.SUCCESS
    w = work(lw.value)
    info = info_buffer(1)
    st = lib.aclsolverSormqr(handle.value, side, trans, m, n, k, da.ptr, da.ld, dt.data_ptr(), dc.ptr, dc.ld,
                             w.data_ptr(), lw.value, info.data_ptr())
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS and int(info.cpu()[0]) == 0
    return dc.read()[0]


@pytest.mark.parametrize("side", [LEFT, RIGHT])
@pytest.mark.parametrize("trans", [OP_N, OP_T, OP_C])
@pytest.mark.parametrize("nq,k,other", [(70, 70, 9), (300, 100, 33), (64, 40, 1)])
def test_sormqr_matches_oracle(handle, side, trans, nq, k, other):
    a = rand(nq, k, nq + k)
    qr, tau = oracle.sgeqrf(a)
    c = rand(nq, other, 3) if side == LEFT else rand(other, nq, 3)
    got = sormqr(handle, side, trans, qr, tau, c)
    assert same_bits(got, oracle.sormqr(side, int(trans != OP_N), qr, tau, c))


@pytest.mark.parametrize("m,n,k", [(100, 80, 60), (64, 64, 64), (50, 20, 0), (300, 300, 257)])
def test_sorgqr_matches_oracle(handle, m, n, k):
    lib = aclsolver.library()
    a = rand(m, max(k, 1), m + n + k)
    qr, tau = oracle.sgeqrf(a)
    tau = tau[:k]
    src = np.zeros((m, n), dtype=np.float32)
    src[:, :k] = qr[:, :k]
    dm = DeviceMatrices(src, m + 2)
    dt = torch.tensor(np.ascontiguousarray(tau) if k else np.zeros(1, np.float32), device="cuda")
    lw = C.c_int(-1)
    assert lib.aclsolverSorgqr_bufferSize(handle.value, m, n, k, dm.ptr, dm.ld, dt.data_ptr(),
                                          C.byref(lw)) == aclsolver.SUCCESS
    w = work(lw.value)
    info = info_buffer(1)
    st = lib.aclsolverSorgqr(handle.value, m, n, k, dm.ptr, dm.ld, dt.data_ptr(), w.data_ptr(), lw.value,
                             info.data_ptr())
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS and int(info.cpu()[0]) == 0
    got = dm.read()[0]
    assert same_bits(got, oracle.sorgqr(src, tau, n))
    assert np.abs(got.T.astype(np.float64) @ got - np.eye(n)).max() < 1e-4


@pytest.mark.parametrize("m,n,nrhs", [(20, 20, 3), (64, 64, 1), (300, 70, 8), (1000, 500, 16), (257, 256, 128)])
def test_sgels_matches_oracle_and_passes_the_gate(handle, m, n, nrhs):
    lib = aclsolver.library()
    a = rand(m, n, m * 3 + n)
    b = rand(m, nrhs, nrhs + 1)
    da = DeviceMatrices(a, m + 1)
    db = DeviceMatrices(b, m + 2)
    dx = DeviceMatrices(np.zeros((n, nrhs), np.float32), n + 3)
    lw = C.c_size_t(0)
    assert lib.aclsolverSSgels_bufferSize(handle.value, m, n, nrhs, da.ptr, da.ld, db.ptr, db.ld, dx.ptr, dx.ld,
                                          None, C.byref(lw)) == aclsolver.SUCCESS
    w = torch.zeros(lw.value // 4 + 1, dtype=torch.float32, device="cuda")
    niter = C.c_int(-5)
    info = info_buffer(1)
    st = lib.aclsolverSSgels(handle.value, m, n, nrhs, da.ptr, da.ld, db.ptr, db.ld, dx.ptr, dx.ld, w.data_ptr(),
                             lw.value, C.byref(niter), info.data_ptr())
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS and int(info.cpu()[0]) == 0 and niter.value == 0
    assert db.unchanged(), "B is read only"
    x = dx.read()[0]
    wx, wqr, _ = oracle.sgels(a.copy(), b)
    assert same_bits(x, wx)
    assert same_bits(da.read()[0], wqr)
    g, gtau = oracle.sgeqr2_golden(a)
    y = oracle.sormqr(0, 1, g, gtau, b)
    xc = np.linalg.solve(np.triu(g[:n, :n]).astype(np.float64), y[:n].astype(np.float64)).astype(np.float32)
    assert judges.gels_ok(a, b, x, xc)


def test_argument_errors_write_info(handle):
    lib = aclsolver.library()
    info = info_buffer(1)
    st = lib.aclsolverSgeqrf(handle.value, 10, 4, None, 9, None, None, 0, info.data_ptr())
    handle.stream.synchronize()
    assert st == 3 and int(info.cpu()[0]) == -4
    st = lib.aclsolverSgeqrf(handle.value, 0, 4, None, 1, None, None, 0, info.data_ptr())
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS and int(info.cpu()[0]) == 0
    a = DeviceMatrices(rand(8, 8, 1), 8)
    st = lib.aclsolverSormqr(handle.value, 0, 1, 8, 8, 9, a.ptr, 8, a.ptr, a.ptr, 8, a.ptr, 1024, info.data_ptr())
    handle.stream.synchronize()
    assert st == 3 and int(info.cpu()[0]) == -5
    niter = C.c_int(7)
    st = lib.aclsolverSSgels(handle.value, 4, 5, 1, a.ptr, 8, a.ptr, 8, a.ptr, 8, a.ptr, 4096, C.byref(niter),
                             info.data_ptr())
    handle.stream.synchronize()
    assert st == 3 and int(info.cpu()[0]) == -1 and niter.value == 0


def xlarft(handle, direct, v, tau, ldt_pad=1):
    lib = aclsolver.library()
    n, k = v.shape
    dv = DeviceMatrices(v, n + 2)
    dtau = torch.tensor(np.ascontiguousarray(tau), device="cuda")
    t0 = np.full((k, k), 9.0, dtype=np.float32)  # the unreferenced triangle must survive
    dt = DeviceMatrices(t0, k + ldt_pad)
    dev, host = C.c_size_t(0), C.c_size_t(1)
    assert lib.aclsolverXlarft_bufferSize(handle.value, None, direct, 0, n, k, 0, dv.ptr, dv.ld, 0, dtau.data_ptr(), 0,
                                          dt.ptr, dt.ld, 0, C.byref(dev), C.byref(host)) == aclsolver.SUCCESS
    assert host.value == 0
    w = torch.empty(dev.value // 4 + 1, dtype=torch.float32, device="cuda")
    st = lib.aclsolverXlarft(handle.value, None, direct, 0, n, k, 0, dv.ptr, dv.ld, 0, dtau.data_ptr(), 0, dt.ptr,
                             dt.ld, 0, w.data_ptr(), dev.value, None, 0)
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS
    return dt.read()[0], t0


@pytest.mark.parametrize("direct", [0, 1])
@pytest.mark.parametrize("n,k", [(1, 1), (40, 7), (100, 32), (300, 33), (1000, 256), (256, 256)])
def test_xlarft_matches_oracle(handle, direct, n, k):
    rng = np.random.default_rng(n + k + direct)
    v = (rng.standard_normal((n, k)) / np.sqrt(n)).astype(np.float32)
    tau = rng.uniform(0.5, 1.5, k).astype(np.float32)
    if k > 3:
        tau[2] = 0.0
    got, t0 = xlarft(handle, direct, v, tau)
    want = oracle.slarft(direct, v, tau, t0)
    assert same_bits(got, want)


def test_xlarft_argument_checks(handle):
    lib = aclsolver.library()
    dev, host = C.c_size_t(0), C.c_size_t(0)
    q = lambda *a: lib.aclsolverXlarft_bufferSize(handle.value, *a, C.byref(dev), C.byref(host))
    assert q(None, 0, 0, 10, 4, 0, None, 10, 0, None, 0, None, 4, 0) == aclsolver.SUCCESS and dev.value == 64
    assert q(C.c_void_p(8), 0, 0, 10, 4, 0, None, 10, 0, None, 0, None, 4, 0) == 3
    assert q(None, 2, 0, 10, 4, 0, None, 10, 0, None, 0, None, 4, 0) == 3
    assert q(None, 0, 0, 3, 4, 0, None, 10, 0, None, 0, None, 4, 0) == 3
    assert q(None, 0, 0, 10, 4, 1, None, 10, 0, None, 0, None, 4, 0) == 7
    assert q(None, 0, 0, 5000, 4, 0, None, 5000, 0, None, 0, None, 4, 0) == 7
    assert q(None, 0, 0, 300, 257, 0, None, 300, 0, None, 0, None, 257, 0) == 7


def test_sgeqrf_captured_in_a_cuda_graph(handle):
    """A call captured on a stream (where the look-ahead's private stream stays off) replays
    to the same bits as the oracle, twice."""
    lib = aclsolver.library()
    m = n = 1024
    a = rand(m, n, 77)
    stream = torch.cuda.Stream()
    with aclsolver.Handle(stream=stream) as h:
        dm = DeviceMatrices(a, m)
        tau = torch.zeros(n, dtype=torch.float32, device="cuda")
        lw = C.c_int(-1)
        assert lib.aclsolverSgeqrf_bufferSize(h.value, m, n, dm.ptr, m, C.byref(lw)) == aclsolver.SUCCESS
        w = work(lw.value)
        info = info_buffer(1)
        original = dm.tensor.clone()

        def call():
            return lib.aclsolverSgeqrf(h.value, m, n, dm.ptr, m, tau.data_ptr(), w.data_ptr(), lw.value,
                                       info.data_ptr())

        assert call() == aclsolver.SUCCESS  # warm-up outside the capture (kernel attributes)
        stream.synchronize()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=stream, capture_error_mode="relaxed"):
            assert call() == aclsolver.SUCCESS
        want, wtau = oracle.sgeqrf(a)
        for _ in range(2):
            dm.tensor.copy_(original)
            torch.cuda.synchronize()
            graph.replay()
            torch.cuda.synchronize()
            assert int(info.cpu()[0]) == 0
            assert same_bits(dm.read()[0], want) and same_bits(tau.cpu().numpy(), wtau)
        del graph


def test_sgeqrf_look_ahead_on_two_streams_at_once():
    """Two handles on two streams factor at the same time; each call forks its own panel
    stream and joins it back, so both results are the oracle's bits."""
    lib = aclsolver.library()
    m, n = 1500, 1200  # tall enough for the look-ahead and the cluster panels
    mats = [rand(m, n, 90 + q) for q in range(2)]
    streams = [torch.cuda.Stream() for _ in range(2)]
    handles = [aclsolver.Handle(stream=s) for s in streams]
    try:
        bufs = []
        for q in range(2):
            dm = DeviceMatrices(mats[q], m + 1)
            tau = torch.zeros(n, dtype=torch.float32, device="cuda")
            lw = C.c_int(-1)
            assert lib.aclsolverSgeqrf_bufferSize(handles[q].value, m, n, dm.ptr, dm.ld, C.byref(lw)) == 0
            bufs.append((dm, tau, work(lw.value), info_buffer(1), lw.value))
        torch.cuda.synchronize()
        for q in range(2):
            dm, tau, w, info, lw = bufs[q]
            assert lib.aclsolverSgeqrf(handles[q].value, m, n, dm.ptr, dm.ld, tau.data_ptr(), w.data_ptr(), lw,
                                       info.data_ptr()) == aclsolver.SUCCESS
        torch.cuda.synchronize()
        for q in range(2):
            dm, tau, _, info, _ = bufs[q]
            want, wtau = oracle.sgeqrf(mats[q])
            assert int(info.cpu()[0]) == 0
            assert same_bits(dm.read()[0], want) and same_bits(tau.cpu().numpy(), wtau)
    finally:
        for h in handles:
            h.close()


@pytest.mark.parametrize("m,n", [(8192, 40), (513, 513), (2049, 97), (600, 1000), (1601, 130), (3000, 64)])
def test_sgeqrf_shape_sweep(handle, m, n):
    """Shapes around the panel thresholds (one block up to 1,600 rows, then an eight-block
    cluster), the look-ahead's (m >= 512, n > 96) and the row limit, against the oracle."""
    a = rand(m, n, m + 7 * n)
    got, tau = geqrf(handle, a, pad=1)
    want, wtau = oracle.sgeqrf(a)
    assert same_bits(tau, wtau) and same_bits(got, want)
