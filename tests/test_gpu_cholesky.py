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


@pytest.mark.parametrize("upper", [False, True])
@pytest.mark.parametrize("n", [1, 5, 8, 9, 32, 33, 100, 129, 300])
def test_spotri_matches_the_solve_of_the_identity(handle, n, upper):
    """aclsolverSpotri: the selected triangle of A^-1 from the factor, in place -- the
    reference's solve of L L^T X = I (cholesky_simt.cpp:220-254) with this build's single
    solve, so bit for bit the oracle's Spotrs on the identity; the other triangle and the
    padding untouched; close to the FP64 inverse."""
    import torch

    lib = aclsolver.library()
    a = spd_batch(1, n, seed=13 * n + int(upper))
    f, winfo = oracle.spotrf_batched(a, upper=upper)
    assert winfo[0] == 0
    tri = np.triu(f[0]) if upper else np.tril(f[0])
    other = np.tril(np.full((n, n), 7.5, dtype=np.float32), -1) if upper else np.triu(np.full((n, n), 7.5, dtype=np.float32), 1)
    dm = DeviceMatrices((tri + other)[None], ld=n + 2)
    lw = C.c_int(-1)
    assert lib.aclsolverSpotri_bufferSize(handle.value, int(upper), n, dm.ptr, dm.ld, C.byref(lw)) == aclsolver.SUCCESS
    work = torch.empty(max(1, lw.value), dtype=torch.float32, device="cuda")
    info = info_buffer(1)
    st = lib.aclsolverSpotri(handle.value, int(upper), n, dm.ptr, dm.ld, work.data_ptr(), lw.value, info.data_ptr())
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS and int(info.cpu()[0]) == 0
    got = dm.read()[0]
    x = oracle.spotrs_batched(f, np.eye(n, dtype=np.float32)[None], upper=upper, single=True)[0]
    want = np.triu(x.T) if upper else np.tril(x)
    got_tri = np.triu(got) if upper else np.tril(got)
    assert same_bits(got_tri, want), first_mismatch(got_tri, want)
    assert np.array_equal(got - got_tri, other), "the other triangle must stay intact"
    inv64 = np.linalg.inv(a[0].astype(np.float64))
    ref_tri = np.triu(inv64) if upper else np.tril(inv64)
    assert np.abs(got_tri - ref_tri).max() <= 1e-4 * np.abs(inv64).max()


def test_spotri_bad_diagonal_leaves_a_unchanged(handle):
    import torch

    lib = aclsolver.library()
    n = 40
    f, _ = oracle.spotrf_batched(spd_batch(1, n, seed=2))
    f = np.tril(f)
    f[0, 17, 17] = -1.0
    dm = DeviceMatrices(f, ld=n)
    work = torch.empty(n * n, dtype=torch.float32, device="cuda")
    info = info_buffer(1)
    st = lib.aclsolverSpotri(handle.value, 0, n, dm.ptr, n, work.data_ptr(), n * n, info.data_ptr())
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS and int(info.cpu()[0]) == 18
    assert dm.unchanged()
    info = info_buffer(1)
    st = lib.aclsolverSpotri(handle.value, 0, n, dm.ptr, n, work.data_ptr(), n * n - 1, info.data_ptr())
    assert st == aclsolver.INVALID_VALUE and int(info.cpu()[0]) == -6


@pytest.mark.parametrize("n,upper", [(257, False), (300, True), (513, False), (1024, False), (2048, False),
                                     (4096, False)])
def test_spotrf_large_matches_oracle(handle, n, upper):
    """Above order 256 one matrix runs over the whole GPU (diagonal block, panel rows and a
    TMA-fed lower-triangle update per 32-column panel): bit for bit the oracle's FMA order."""
    lib = aclsolver.library()
    a = spd_batch(1, n, seed=n + int(upper))
    da = DeviceMatrices(a, ld=n + (4 if n % 2 == 0 else 1))
    info = info_buffer(1)
    st = lib.aclsolverSpotrf(handle.value, int(upper), n, da.ptr, da.ld, None, 0, info.data_ptr())
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS and int(info.cpu()[0]) == 0
    want, winfo = oracle.spotrf_batched(a, upper=upper)
    got = da.read()
    tri = (lambda m: np.triu(m)) if upper else (lambda m: np.tril(m))
    assert same_bits(tri(got[0]), tri(want[0])), first_mismatch(tri(got[0]), tri(want[0]))
    assert np.array_equal(got[0] - tri(got[0]), a[0] - tri(a[0])), "the other triangle must stay intact"


@pytest.mark.parametrize("n,bad", [(300, 100), (300, 290), (520, 33), (520, 511)])
def test_spotrf_large_failure_keeps_unfinished_columns(handle, n, bad):
    lib = aclsolver.library()
    a = spd_batch(1, n, seed=4)
    a[0, bad, bad] = -1.0
    da = DeviceMatrices(a, ld=n)
    info = info_buffer(1)
    st = lib.aclsolverSpotrf(handle.value, 0, n, da.ptr, n, None, 0, info.data_ptr())
    handle.stream.synchronize()
    want, winfo = oracle.spotrf_batched(a)
    assert st == aclsolver.SUCCESS and int(info.cpu()[0]) == int(winfo[0]) > 0
    got = da.read()
    assert same_bits(np.tril(got[0]), np.tril(want[0])), first_mismatch(np.tril(got[0]), np.tril(want[0]))


def test_spotrf_batched_above_packed_orders(handle):
    a = spd_batch(3, 300, seed=12)
    a[1, 150, 150] = 0.0
    st, dm, info = potrf_batched(handle, a, False)
    want, winfo = oracle.spotrf_batched(a)
    assert st == aclsolver.SUCCESS and info.tolist() == winfo.tolist()
    assert same_bits(np.tril(dm.read()), np.tril(want))


@pytest.mark.parametrize("n", [1024, 2048, 4096])
def test_large_spotrf_spotrs_pass_the_reference_residual_gate(handle, n):
    """The reference's residual judge (test/cholesky/lapack_residual.py: ratio <= 5 x FP32
    LAPACK's) at the orders where a plain ascending-k chain of n roundings per element fails
    it: the whole-GPU factor and the blocked solve take each 64-column panel as one partial
    sum, which keeps them near LAPACK's ratio.  Bit for bit the oracle's order where the
    oracle finishes in seconds (n <= 2048)."""
    lib = aclsolver.library()
    a = spd_batch(1, n, seed=n + 5)
    da = DeviceMatrices(a, ld=n)
    info = info_buffer(1)
    st = lib.aclsolverSpotrf(handle.value, 0, n, da.ptr, n, None, 0, info.data_ptr())
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS and int(info.cpu()[0]) == 0
    f = da.read()
    b = np.random.default_rng(n).standard_normal((1, n, 1)).astype(np.float32)
    db = DeviceMatrices(b, ld=n)
    st = lib.aclsolverSpotrs(handle.value, 0, n, 1, da.ptr, n, db.ptr, n, info.data_ptr())
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS and int(info.cpu()[0]) == 0
    x = db.read()
    if n <= 2048:
        wf, _ = oracle.spotrf_batched(a)
        assert same_bits(np.tril(f[0]), np.tril(wf[0]))
        assert same_bits(x, oracle.spotrs_batched(wf, b, single=True))
    r, c = judges.paired_cholesky("potrf", a[0], f[0])
    assert r <= 5 * c, (r, c)
    rs, cs = judges.paired_cholesky("potrs", a[0], x[0], b32=b[0])
    assert rs <= 5 * cs, (rs, cs)
