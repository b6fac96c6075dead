"""Blocked real LU (64 < n <= 512) and the blocked LU solve through the C ABI on the GPU:
identical ipiv and info, bit-identical factors and solutions against the oracle's unblocked
order (orc_sgetrf / orc_sgetrs), at sizes that exercise ragged panels and tiles."""

import ctypes as C

import numpy as np
import pytest

import aclsolver
import oracle
from oracle import judges
from helpers import DeviceMatrices, device_ints, first_mismatch, info_buffer, same_bits

pytestmark = pytest.mark.gpu


def gaussian(count, n, seed, m=None):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((count, m or n, n)).astype(np.float32)


def getrf_batched(handle, a, pivoting=True, pad=3):
    lib = aclsolver.library()
    count, n, _ = a.shape
    dm = DeviceMatrices(a, ld=n + pad)
    piv = device_ints(np.zeros(count * n)) if pivoting else None
    info = info_buffer(count)
    st = lib.aclsolverSgetrfBatched(handle.value, n, dm.table_ptr, dm.ld, None if piv is None else piv.data_ptr(),
                                   info.data_ptr(), count)
    handle.stream.synchronize()
    ipiv = piv.cpu().numpy().reshape(count, n) if pivoting else None
    return st, dm, ipiv, info.cpu().numpy()


@pytest.mark.parametrize("n", [65, 96, 100, 127, 128, 129, 160, 200, 255, 256, 257, 333, 384, 500, 512])
def test_blocked_sgetrf_matches_oracle(handle, n):
    a = gaussian(3, n, seed=1000 + n)
    st, dm, ipiv, info = getrf_batched(handle, a)
    assert st == aclsolver.SUCCESS
    lu, wpiv, winfo = oracle.sgetrf_batched(a)
    assert info.tolist() == winfo.tolist()
    assert np.array_equal(ipiv, wpiv), "pivot sequences differ"
    got = dm.read()
    assert same_bits(got, lu), first_mismatch(got, lu)


@pytest.mark.parametrize("n", [100, 200])
def test_blocked_sgetrf_integer_ties(handle, n):
    """Small integers (randint 1..10) force exact pivot ties: the earliest row must win."""
    rng = np.random.default_rng(n)
    a = rng.integers(1, 11, size=(2, n, n)).astype(np.float32)
    st, dm, ipiv, info = getrf_batched(handle, a)
    lu, wpiv, winfo = oracle.sgetrf_batched(a)
    assert info.tolist() == winfo.tolist()
    assert np.array_equal(ipiv, wpiv)
    assert same_bits(dm.read(), lu)


def test_blocked_sgetrf_special_values(handle):
    n = 150
    a = gaussian(5, n, seed=77)
    a[0, :, 70] = 0.0  # zero column inside the third panel: info 71, factorisation continues
    a[1, 90, 90] = np.nan
    a[2, 10, 3] = np.inf
    a[3] *= 1e-39  # subnormal entries
    a[4, :, 0] = 2.0  # all-equal first column: earliest row wins
    st, dm, ipiv, info = getrf_batched(handle, a)
    lu, wpiv, winfo = oracle.sgetrf_batched(a)
    assert info.tolist() == winfo.tolist()
    assert info[0] == 71
    assert np.array_equal(ipiv, wpiv)
    assert same_bits(dm.read(), lu), first_mismatch(dm.read(), lu)


def test_blocked_sgetrf_zero_pivot_without_pivoting(handle):
    """Without pivoting a zero U(k,k) leaves a nonzero L column below it, which must take no
    part in later updates (panel, triangular solve and trailing tiles)."""
    n = 140
    a = gaussian(2, n, seed=5) + 4 * np.eye(n, dtype=np.float32)
    a[0, :40, 40:] = 0.0  # the trailing block after 40 steps is exactly A[40:, 40:]
    a[0, 40, 40] = 0.0  # -> U(40, 40) = 0 with A[41:, 40] nonzero
    a[1, 0, 0] = 0.0  # first pivot zero
    st, dm, _, info = getrf_batched(handle, a, pivoting=False)
    lu, _, winfo = oracle.sgetrf_batched(a, pivoting=False)
    assert st == aclsolver.SUCCESS
    assert info.tolist() == winfo.tolist() == [41, 1]
    assert same_bits(dm.read(), lu), first_mismatch(dm.read(), lu)


def test_blocked_sgetrf_batch_of_512(handle):
    """64 matrices of 512 x 512 (the mixed-precision workload's order): exact parity."""
    a = gaussian(64, 512, seed=3)
    st, dm, ipiv, info = getrf_batched(handle, a, pad=0)
    lu, wpiv, winfo = oracle.sgetrf_batched(a)
    assert st == aclsolver.SUCCESS and np.all(info == 0)
    assert np.array_equal(ipiv, wpiv)
    assert same_bits(dm.read(), lu)
    assert judges.lu_reconstruction_ok(a[0], dm.read()[0], wpiv[0])


def test_blocked_sgetrf_null_slot(handle):
    lib = aclsolver.library()
    n = 80
    a = gaussian(3, n, seed=8)
    dm = DeviceMatrices(a, ld=n)
    table = dm.table.clone()
    table[1] = 0
    piv = device_ints(np.zeros(3 * n))
    info = info_buffer(3)
    st = lib.aclsolverSgetrfBatched(handle.value, n, table.data_ptr(), n, piv.data_ptr(), info.data_ptr(), 3)
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS
    assert info.cpu().tolist() == [0, -2, 0]
    lu, wpiv, _ = oracle.sgetrf_batched(a[[0, 2]])
    got = dm.read()
    assert same_bits(got[[0, 2]], lu)
    assert np.array_equal(got[1], a[1])


@pytest.mark.parametrize("m,n", [(300, 300), (65, 65)])
def test_blocked_sgetrf_single(handle, m, n):
    import torch

    lib = aclsolver.library()
    a = gaussian(1, n, seed=m + 5, m=m)
    dm = DeviceMatrices(a, ld=m + 1)
    lw = C.c_int(-1)
    assert lib.aclsolverSgetrf_bufferSize(handle.value, m, n, dm.ptr, dm.ld, C.byref(lw)) == aclsolver.SUCCESS
    work = torch.empty(max(1, lw.value), dtype=torch.float32, device="cuda")
    piv = device_ints(np.zeros(n))
    info = info_buffer(1)
    st = lib.aclsolverSgetrf(handle.value, m, n, dm.ptr, dm.ld, work.data_ptr(), piv.data_ptr(), info.data_ptr())
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS
    lu, wpiv, winfo = oracle.sgetrf_batched(a)
    assert int(info.cpu()[0]) == winfo[0]
    assert piv.cpu().tolist() == wpiv[0].tolist()
    assert same_bits(dm.read(), lu)


def getrs_batched(handle, lu, ipiv, b, pad=1, trans=0):
    lib = aclsolver.library()
    count, n, _ = lu.shape
    da = DeviceMatrices(lu, ld=n + pad)
    db = DeviceMatrices(b, ld=n + pad + 1)
    piv = None if ipiv is None else device_ints(ipiv.reshape(-1))
    info = info_buffer(count)
    st = lib.aclsolverSgetrsBatched(handle.value, trans, n, b.shape[2], da.table_ptr, da.ld,
                                   None if piv is None else piv.data_ptr(), db.table_ptr, db.ld, info.data_ptr(),
                                   count)
    handle.stream.synchronize()
    return st, da, db, info.cpu().numpy()


@pytest.mark.parametrize("n,nrhs", [(65, 1), (100, 3), (128, 8), (200, 9), (512, 1), (512, 16), (1000, 2)])
def test_blocked_sgetrs_matches_oracle(handle, n, nrhs):
    a = gaussian(3, n, seed=n + 11)
    lu, ipiv, _ = oracle.sgetrf_batched(a)
    b = gaussian(3, nrhs, seed=n + 12, m=n)
    st, da, db, info = getrs_batched(handle, lu, ipiv, b)
    assert st == aclsolver.SUCCESS and np.all(info == 0)
    assert da.unchanged()
    want = oracle.sgetrs_batched(lu, ipiv, b)
    got = db.read()
    assert same_bits(got, want), first_mismatch(got, want)
    assert judges.solve_compare_ok(got[0], judges.solve_lu(lu[0], b[0], ipiv[0], 0))


@pytest.mark.parametrize("n,nrhs,pad", [(65, 1, 1), (96, 2, 0), (100, 3, 1), (225, 4, 3), (513, 9, 0), (1000, 2, 1),
                                        (2049, 1, 0)])
def test_blocked_sgetrs_transposed_matches_oracle(handle, n, nrhs, pad):
    """A^T x = b above the register-resident orders: U^T forward, L^T backward, then the
    interchanges in reverse, bit for bit the oracle's order (strips of 224 factor columns,
    ragged last blocks, 16-byte and 4-byte staging)."""
    a = gaussian(2, n, seed=n + 21)
    lu, ipiv, _ = oracle.sgetrf_batched(a)
    b = gaussian(2, nrhs, seed=n + 22, m=n)
    st, da, db, info = getrs_batched(handle, lu, ipiv, b, pad=pad, trans=1)
    assert st == aclsolver.SUCCESS and np.all(info == 0)
    assert da.unchanged()
    want = oracle.sgetrs_batched(lu, ipiv, b, trans=1)
    got = db.read()
    assert same_bits(got, want), first_mismatch(got, want)
    assert judges.solve_compare_ok(got[1], judges.solve_lu(lu[1], b[1], ipiv[1], 1))


def test_blocked_sgetrs_transposed_without_pivots_and_bad_pivot(handle):
    n = 130
    a = gaussian(2, n, seed=7) + 6 * np.eye(n, dtype=np.float32)
    lu, _, _ = oracle.sgetrf_batched(a, pivoting=False)
    b = gaussian(2, 2, seed=8, m=n)
    st, _, db, info = getrs_batched(handle, lu, None, b, trans=1)
    assert st == aclsolver.SUCCESS and np.all(info == 0)
    assert same_bits(db.read(), oracle.sgetrs_batched(lu, None, b, trans=1))
    lu, ipiv, _ = oracle.sgetrf_batched(a)
    ipiv = ipiv.copy()
    ipiv[1, 77] = 0  # below 1
    st, _, db, info = getrs_batched(handle, lu, ipiv, b, trans=1)
    assert info.tolist() == [0, -6]
    assert np.array_equal(db.read()[1], b[1])
    assert same_bits(db.read()[0], oracle.sgetrs_batched(lu[:1], ipiv[:1], b[:1], trans=1)[0])


def test_blocked_sgetrs_without_pivots(handle):
    n = 130
    a = gaussian(2, n, seed=4) + 6 * np.eye(n, dtype=np.float32)
    lu, _, _ = oracle.sgetrf_batched(a, pivoting=False)
    b = gaussian(2, 2, seed=6, m=n)
    st, _, db, info = getrs_batched(handle, lu, None, b)
    assert st == aclsolver.SUCCESS and np.all(info == 0)
    assert same_bits(db.read(), oracle.sgetrs_batched(lu, None, b))


def test_blocked_sgetrs_bad_pivot(handle):
    n = 96
    a = gaussian(3, n, seed=1)
    lu, ipiv, _ = oracle.sgetrf_batched(a)
    ipiv = ipiv.copy()
    ipiv[2, 50] = n + 1  # above n
    b = gaussian(3, 1, seed=2, m=n)
    st, _, db, info = getrs_batched(handle, lu, ipiv, b)
    assert info.tolist() == [0, 0, -6]
    assert np.array_equal(db.read()[2], b[2])


@pytest.mark.parametrize("n,nrhs,trans", [(100, 1, 0), (520, 3, 0), (100, 2, 1), (520, 3, 1)])
def test_blocked_sgetrs_host_buffers(handle, n, nrhs, trans):
    """The host-buffer, row-major aclsolverSgetrs above the register-resident orders, both
    trans codes."""
    lib = aclsolver.library()
    a = gaussian(1, n, seed=n)
    lu, ipiv, _ = oracle.sgetrf_batched(a)
    b = gaussian(1, nrhs, seed=n + 1, m=n)[0]
    lda, ldb = n + 2, nrhs + 1
    A = np.zeros((n, lda), dtype=np.float32)
    A[:, :n] = lu[0]
    B = np.full((n, ldb), 3.25, dtype=np.float32)
    B[:, :nrhs] = b
    P = np.ascontiguousarray(ipiv[0], dtype=np.int32)
    info = np.array([99], dtype=np.int32)
    st = lib.aclsolverSgetrs(handle.value, trans, n, nrhs, A.ctypes.data, lda, P.ctypes.data, B.ctypes.data, ldb,
                             info.ctypes.data)
    assert st == 0 and info[0] == 0
    assert np.all(B[:, nrhs:] == 3.25)
    want = oracle.sgetrs_batched(lu, ipiv, b[None], trans=trans)[0]
    assert same_bits(B[:, :nrhs], want), first_mismatch(B[:, :nrhs], want)
