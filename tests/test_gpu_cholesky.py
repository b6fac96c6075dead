"""Real Cholesky parity through the C ABI on the GPU: SpotrfBatched, SpotrsBatched,
Spotrf, Spotrs against the oracle, bit for bit, plus the reference's contracts (padding
and the unselected triangle untouched, per-slot info, null slots, failed pivots)."""

import ctypes as C

import numpy as np
import pytest

import aclsolver
import oracle
from oracle import judges
from helpers import (
    DeviceMatrices,
    POISON,
    first_mismatch,
    info_buffer,
    same_bits,
    spd_batch,
)

pytestmark = pytest.mark.gpu

SIZES = [1, 2, 5, 8, 9, 12, 16, 17, 24, 31, 32, 33, 48, 64, 65, 100, 128, 129, 200]


def potrf_batched(handle, a, upper, pad=3):
    lib = aclsolver.library()
    count, n, _ = a.shape
    dm = DeviceMatrices(a, ld=n + pad)
    info = info_buffer(count)
    st = lib.aclsolverSpotrfBatched(handle.value, int(upper), n, dm.table_ptr, dm.ld, info.data_ptr(), count)
    handle.stream.synchronize()
    return st, dm, info.cpu().numpy()


@pytest.mark.parametrize("upper", [False, True])
@pytest.mark.parametrize("n", SIZES)
def test_spotrf_batched_matches_oracle(handle, n, upper):
    a = spd_batch(7, n, seed=n)
    st, dm, info = potrf_batched(handle, a, upper)
    assert st == aclsolver.SUCCESS
    assert np.all(info == 0)
    got = dm.read()
    want, winfo = oracle.spotrf_batched(a, upper=upper)
    assert np.all(winfo == 0)
    assert same_bits(got, want), first_mismatch(got, want)


def test_spotrf_batched_config_size(handle):
    """10,000 SPD 32x32 matrices A = G G^T/32 + I (the batched Cholesky workload)."""
    a = spd_batch(10000, 32, seed=0)
    st, dm, info = potrf_batched(handle, a, False, pad=0)
    assert st == aclsolver.SUCCESS and np.all(info == 0)
    want, _ = oracle.spotrf_batched(a)
    assert same_bits(dm.read(), want)


@pytest.mark.parametrize("n", [4, 12, 32, 40])
def test_spotrf_batched_failure_keeps_unfinished_columns(handle, n):
    a = spd_batch(4, n, seed=3)
    k = n // 2
    a[1, k, k] = -50.0
    a[2, n - 1, n - 1] = np.nan
    st, dm, info = potrf_batched(handle, a, False)
    want, winfo = oracle.spotrf_batched(a)
    assert st == aclsolver.SUCCESS
    assert info.tolist() == winfo.tolist()
    assert info[1] > 0 and info[2] > 0 and info[0] == 0 and info[3] == 0
    assert same_bits(dm.read(), want)


def test_spotrf_batched_null_slot(handle):
    lib = aclsolver.library()
    a = spd_batch(3, 16, seed=5)
    dm = DeviceMatrices(a, ld=16)
    dm.table[1] = 0
    info = info_buffer(3)
    st = lib.aclsolverSpotrfBatched(handle.value, 0, 16, dm.table_ptr, 16, info.data_ptr(), 3)
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS
    assert info.cpu().tolist() == [0, -3, 0]
    assert np.array_equal(dm.read()[1], a[1])


@pytest.mark.parametrize(
    "args,code",
    [
        ((2, 4, True, 4, 2), -1),  # bad uplo
        ((0, 4097, True, 4097, 2), -2),  # n too large
        ((0, 4, False, 4, 2), -3),  # null pointer table
        ((0, 4, True, 3, 2), -4),  # lda < n
    ],
)
def test_spotrf_batched_argument_errors_fill_every_slot(handle, args, code):
    lib = aclsolver.library()
    uplo, n, table, lda, count = args
    dm = DeviceMatrices(spd_batch(2, 4, seed=1), ld=4)
    info = info_buffer(count)
    st = lib.aclsolverSpotrfBatched(handle.value, uplo, n, dm.table_ptr if table else None, lda, info.data_ptr(),
                                   count)
    handle.stream.synchronize()
    assert st == aclsolver.INVALID_VALUE
    assert info.cpu().tolist() == [code] * count


def test_spotrf_batched_empty_problems(handle):
    lib = aclsolver.library()
    info = info_buffer(3)
    assert lib.aclsolverSpotrfBatched(handle.value, 0, 0, None, 1, info.data_ptr(), 3) == aclsolver.SUCCESS
    handle.stream.synchronize()
    assert info.cpu().tolist() == [0, 0, 0]
    assert lib.aclsolverSpotrfBatched(handle.value, 0, 4, None, 4, None, 0) == aclsolver.SUCCESS


def potrs_batched(handle, factors, b, upper, pad=2):
    lib = aclsolver.library()
    count, n, _ = factors.shape
    da = DeviceMatrices(factors, ld=n + pad)
    db = DeviceMatrices(b, ld=n + pad)
    info = info_buffer(1)
    st = lib.aclsolverSpotrsBatched(handle.value, int(upper), n, 1, da.table_ptr, da.ld, db.table_ptr, db.ld,
                                   info.data_ptr(), count)
    handle.stream.synchronize()
    return st, da, db, int(info.cpu()[0])


@pytest.mark.parametrize("upper", [False, True])
@pytest.mark.parametrize("n", SIZES)
def test_spotrs_batched_matches_oracle(handle, n, upper):
    a = spd_batch(6, n, seed=100 + n)
    f, _ = oracle.spotrf_batched(a, upper=upper)
    b = np.random.default_rng(n).standard_normal((6, n, 1)).astype(np.float32)
    st, da, db, info = potrs_batched(handle, f, b, upper)
    assert st == aclsolver.SUCCESS and info == 0
    assert da.unchanged(), "factor modified by the solve"
    want = oracle.spotrs_batched(f, b, upper=upper)
    got = db.read()
    assert same_bits(got, want), first_mismatch(got, want)
    ok, _, bad = judges.cholesky_batch_passes("potrs", a, got, upper, b)
    assert ok, bad


def test_factor_then_solve_config_size(handle):
    """10,000 x (32x32 factor + 1 RHS) through both entry points, bitwise and judged."""
    a = spd_batch(10000, 32, seed=0)
    b = np.random.default_rng(0).standard_normal((10000, 32, 1)).astype(np.float32)
    st, dm, info = potrf_batched(handle, a, False, pad=0)
    f = dm.read()
    st2, _, db, info2 = potrs_batched(handle, f, b, False, pad=0)
    assert st == st2 == aclsolver.SUCCESS and info2 == 0
    wf, _ = oracle.spotrf_batched(a)
    wx = oracle.spotrs_batched(wf, b)
    assert same_bits(f, wf)
    assert same_bits(db.read(), wx)
    sample = np.arange(0, 10000, 97)
    ok, _, bad = judges.cholesky_batch_passes("potrs", a[sample], db.read()[sample], False, b[sample])
    assert ok, bad


@pytest.mark.parametrize("slot,code", [("a", -4), ("b", -6)])
def test_spotrs_batched_null_slot_contract(handle, slot, code):
    lib = aclsolver.library()
    n = 8
    f, _ = oracle.spotrf_batched(spd_batch(3, n, seed=2))
    b = np.ones((3, n, 1), dtype=np.float32)
    da, db = DeviceMatrices(f, ld=n), DeviceMatrices(b, ld=n)
    (da if slot == "a" else db).table[2] = 0
    info = info_buffer(1)
    st = lib.aclsolverSpotrsBatched(handle.value, 0, n, 1, da.table_ptr, n, db.table_ptr, n, info.data_ptr(), 3)
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS
    assert int(info.cpu()[0]) == code
    assert db.unchanged(), "right-hand sides must stay intact on slot errors"


@pytest.mark.parametrize("n,nrhs", [(1, 1), (6, 3), (8, 5), (16, 2), (33, 4), (64, 1), (128, 3), (150, 2)])
def test_spotrf_spotrs_single(handle, n, nrhs):
    lib = aclsolver.library()
    a = spd_batch(1, n, seed=7 * n)
    da = DeviceMatrices(a, ld=n + 1)
    lw = C.c_int(-1)
    assert lib.aclsolverSpotrf_bufferSize(handle.value, 0, n, da.ptr, da.ld, C.byref(lw)) == aclsolver.SUCCESS
    info = info_buffer(1)
    st = lib.aclsolverSpotrf(handle.value, 0, n, da.ptr, da.ld, None, 0, info.data_ptr())
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS and int(info.cpu()[0]) == 0
    f = da.read()
    wf, _ = oracle.spotrf_batched(a)
    assert same_bits(f, wf)
    b = np.random.default_rng(n).standard_normal((1, n, nrhs)).astype(np.float32)
    db = DeviceMatrices(b, ld=n + 2)
    st = lib.aclsolverSpotrs(handle.value, 0, n, nrhs, da.ptr, da.ld, db.ptr, db.ld, info.data_ptr())
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS and int(info.cpu()[0]) == 0
    want = oracle.spotrs_batched(wf, b, single=True)
    assert same_bits(db.read(), want), first_mismatch(db.read(), want)


def test_repeat_calls_are_bitwise_identical(handle):
    a = spd_batch(64, 24, seed=11)
    outs = []
    for _ in range(3):
        st, dm, info = potrf_batched(handle, a, False)
        outs.append(dm.read())
    assert same_bits(outs[0], outs[1]) and same_bits(outs[1], outs[2])
