"""Two batched entries above their register-resident orders: aclsolverSgetriBatched for
64 < n (inverse as the blocked solve against the identity; tolerance against the oracle's
vector-inverse order and FP64), and aclsolverSgetrfBatched above 512 (each matrix over the
whole GPU: bit for bit with the oracle)."""

import numpy as np
import pytest
import torch

import aclsolver
import oracle
from helpers import DeviceMatrices, device_ints, first_mismatch, info_buffer, same_bits

pytestmark = pytest.mark.gpu


def gaussian(count, n, seed):
    return np.random.default_rng(seed).standard_normal((count, n, n)).astype(np.float32)


def getri(handle, lu, ipiv, pad=2, null_slot=None):
    lib = aclsolver.library()
    count, n, _ = lu.shape
    da = DeviceMatrices(lu, ld=n + 1)
    dc = DeviceMatrices(np.full_like(lu, 7.0), ld=n + pad)
    ctab = dc.table.clone()
    if null_slot is not None:
        ctab[null_slot] = 0
    piv = None if ipiv is None else device_ints(ipiv.reshape(-1))
    info = info_buffer(count)
    st = lib.aclsolverSgetriBatched(handle.value, n, da.table_ptr, da.ld, None if piv is None else piv.data_ptr(),
                                   ctab.data_ptr(), dc.ld, info.data_ptr(), count)
    handle.stream.synchronize()
    return st, dc.read(), info.cpu().numpy()


@pytest.mark.parametrize("n", [65, 100, 200, 512])
def test_getri_blocked_matches_oracle_and_fp64(handle, n):
    a = gaussian(3, n, seed=n) + 3 * np.eye(n, dtype=np.float32)
    lu, ipiv, _ = oracle.sgetrf_batched(a)
    st, c, info = getri(handle, lu, ipiv)
    assert st == aclsolver.SUCCESS and np.all(info == 0)
    want, winfo = oracle.sgetri_batched(lu, ipiv)
    assert np.all(winfo == 0)
    for q in range(3):
        inv64 = np.linalg.inv(a[q].astype(np.float64))
        scale = np.abs(inv64).max()
        assert np.abs(c[q] - want[q]).max() <= 1e-4 * scale
        assert np.abs(c[q] - inv64).max() <= 1e-4 * scale
        assert np.abs(a[q].astype(np.float64) @ c[q] - np.eye(n)).max() <= 1e-4 * n


def test_getri_blocked_info_conventions(handle):
    """With the synchronous checks off (they refuse such input up front, as the reference
    does): null C slot -2, bad pivot -4, zero U diagonal k+1 (C left as it was), others
    solved."""
    lib = aclsolver.library()
    n = 96
    a = gaussian(4, n, seed=5) + 3 * np.eye(n, dtype=np.float32)
    lu, ipiv, _ = oracle.sgetrf_batched(a)
    lu = lu.copy()
    ipiv = ipiv.copy()
    ipiv[1, 10] = n + 3
    lu[2, 40, 40] = 0.0
    st, _, info = getri(handle, lu, ipiv, null_slot=0)
    assert st == aclsolver.INVALID_VALUE  # the checks catch the null slot first
    aclsolver.check(lib.aclsolverSetDeviceChecks(handle.value, 0))
    try:
        st, c, info = getri(handle, lu, ipiv, null_slot=0)
    finally:
        aclsolver.check(lib.aclsolverSetDeviceChecks(handle.value, 1))
    assert st == aclsolver.SUCCESS
    assert info.tolist() == [-2, -4, 41, 0]
    assert np.all(c[1] == 7.0) and np.all(c[2] == 7.0)
    inv64 = np.linalg.inv(a[3].astype(np.float64))
    assert np.abs(c[3] - inv64).max() <= 1e-4 * np.abs(inv64).max()


def test_getri_blocked_without_pivots(handle):
    n = 130
    a = gaussian(2, n, seed=9) + 20 * np.eye(n, dtype=np.float32)
    lu, _, _ = oracle.sgetrf_batched(a, pivoting=False)
    st, c, info = getri(handle, lu, None)
    assert st == aclsolver.SUCCESS and np.all(info == 0)
    for q in range(2):
        inv64 = np.linalg.inv(a[q].astype(np.float64))
        assert np.abs(c[q] - inv64).max() <= 1e-4 * np.abs(inv64).max()


def test_sgetrf_batched_above_512_matches_oracle(handle):
    lib = aclsolver.library()
    n, count = 600, 3
    a = gaussian(count, n, seed=17)
    dm = DeviceMatrices(a, ld=n + 3)
    table = dm.table.clone()
    table[1] = 0  # a null slot: info -2, the others factored
    piv = device_ints(np.zeros(count * n))
    info = info_buffer(count)
    st = lib.aclsolverSgetrfBatched(handle.value, n, table.data_ptr(), dm.ld, piv.data_ptr(), info.data_ptr(), count)
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS
    assert info.cpu().tolist() == [0, -2, 0]
    lu, wpiv, _ = oracle.sgetrf_batched(a[[0, 2]])
    got = dm.read()
    ipiv = piv.cpu().numpy().reshape(count, n)
    assert np.array_equal(ipiv[[0, 2]], wpiv)
    assert same_bits(got[[0, 2]], lu), first_mismatch(got[[0, 2]], lu)
    assert np.array_equal(got[1], a[1])


@pytest.mark.parametrize("n,pivoting", [(65, True), (200, True), (129, False), (1000, True)])
def test_getri_single_above_small_orders(handle, n, pivoting):
    """aclsolverSgetri (in place, caller workspace) above order 64: the factors copied to the
    workspace, A solved against the identity; tolerance against the oracle's inverse and
    FP64, the workspace query and info conventions of the small path."""
    import ctypes as C

    lib = aclsolver.library()
    # without pivoting, a diagonally dominant matrix keeps the factors' growth small
    a = gaussian(1, n, seed=3 * n) + (3 if pivoting else 2 * n) * np.eye(n, dtype=np.float32)
    lu, ipiv, _ = oracle.sgetrf_batched(a, pivoting=pivoting)
    dm = DeviceMatrices(lu, ld=n + 3)
    lw = C.c_int(-1)
    assert lib.aclsolverSgetri_bufferSize(handle.value, n, dm.ptr, dm.ld, C.byref(lw)) == aclsolver.SUCCESS
    assert lw.value >= n * n
    work = torch.empty(lw.value, dtype=torch.float32, device="cuda")
    piv = device_ints(ipiv[0]) if pivoting else None
    info = info_buffer(1)
    st = lib.aclsolverSgetri(handle.value, n, dm.ptr, dm.ld, None if piv is None else piv.data_ptr(),
                             work.data_ptr(), lw.value, info.data_ptr())
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS and int(info.cpu()[0]) == 0
    got = dm.read()[0]
    want, _ = oracle.sgetri_batched(lu, ipiv if pivoting else None)
    scale = np.abs(want[0]).max()
    assert np.abs(got - want[0]).max() <= 1e-4 * scale

    # the reference's inverse residual gate: ||I - A X||_1 / (n ||A||_1 ||X||_1 eps) within
    # max(5 x the FP32 oracle's ratio, 0.1) (test/cholesky/lapack_residual.py, INVERSE floor)
    def ratio(x):
        a64, x64 = a[0].astype(np.float64), x.astype(np.float64)
        norm1 = lambda m: np.abs(m).sum(axis=0).max()
        return norm1(np.eye(n) - a64 @ x64) / (n * norm1(a64) * norm1(x64) * np.finfo(np.float32).eps)

    assert ratio(got) <= max(5 * ratio(want[0]), 0.1)


def test_getri_single_zero_diagonal(handle):
    import ctypes as C

    lib = aclsolver.library()
    aclsolver.check(lib.aclsolverSetDeviceChecks(handle.value, 0))
    n = 100
    a = gaussian(1, n, seed=8) + 3 * np.eye(n, dtype=np.float32)
    lu, ipiv, _ = oracle.sgetrf_batched(a)
    lu[0, 40, 40] = 0.0
    dm = DeviceMatrices(lu, ld=n)
    work = torch.empty(n * n, dtype=torch.float32, device="cuda")
    piv = device_ints(ipiv[0])
    info = info_buffer(1)
    st = lib.aclsolverSgetri(handle.value, n, dm.ptr, n, piv.data_ptr(), work.data_ptr(), n * n, info.data_ptr())
    handle.stream.synchronize()
    aclsolver.check(lib.aclsolverSetDeviceChecks(handle.value, 1))
    assert st == aclsolver.SUCCESS and int(info.cpu()[0]) == 41
    assert dm.unchanged(), "a singular factor is left as it was"
