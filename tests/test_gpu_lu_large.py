"""aclsolverSgetrf above the batched-blocked orders: one matrix over the whole GPU (cluster
panels, 128-column outer blocks).  Pivots, info and factors equal the oracle's unblocked order
bit for bit up to order 2048; at 8192, where the scalar oracle would take hours, the factors are
judged by the FP64 backward error of the solve they give and by the pivot sequence's range."""

import ctypes as C

import numpy as np
import pytest
import scipy.linalg as sla
import torch

import aclsolver
import oracle
from oracle import judges
from helpers import DeviceMatrices, conditioned_batch, device_ints, first_mismatch, info_buffer, same_bits

pytestmark = pytest.mark.gpu


def sgetrf(handle, a, pad=1, pivoting=True):
    lib = aclsolver.library()
    m, n = a.shape
    dm = DeviceMatrices(a[None], ld=m + pad)
    lw = C.c_int(-1)
    assert lib.aclsolverSgetrf_bufferSize(handle.value, m, n, dm.ptr, dm.ld, C.byref(lw)) == aclsolver.SUCCESS
    work = torch.empty(max(1, lw.value), dtype=torch.float32, device="cuda")
    piv = device_ints(np.zeros(min(m, n))) if pivoting else None
    info = info_buffer(1)
    st = lib.aclsolverSgetrf(handle.value, m, n, dm.ptr, dm.ld, work.data_ptr(),
                             None if piv is None else piv.data_ptr(), info.data_ptr())
    handle.stream.synchronize()
    ipiv = piv.cpu().numpy() if pivoting else None
    return st, dm.read()[0], ipiv, int(info.cpu()[0])


def gaussian(m, n, seed):
    return np.random.default_rng(seed).standard_normal((m, n)).astype(np.float32)


@pytest.mark.parametrize("m,n", [(513, 513), (640, 640), (1000, 1000), (700, 300), (1030, 520), (600, 512),
                                 (2048, 2048)])
def test_large_sgetrf_matches_oracle(handle, m, n):
    a = gaussian(m, n, seed=m * 7 + n)
    st, got, ipiv, info = sgetrf(handle, a)
    assert st == aclsolver.SUCCESS
    lu, wpiv, winfo = oracle.sgetrf_batched(a[None])
    assert info == winfo[0] == 0
    assert np.array_equal(ipiv, wpiv[0]), "pivot sequences differ"
    assert same_bits(got, lu[0]), first_mismatch(got, lu[0])


def test_large_sgetrf_zero_column_and_ties(handle):
    """A zero column (info, and a column that takes no part in later updates) and exact ties
    from small integers (the earliest row wins), in one 700 x 700 matrix."""
    n = 700
    rng = np.random.default_rng(11)
    a = rng.integers(1, 9, size=(n, n)).astype(np.float32)
    a[:, 200] = 0.0
    st, got, ipiv, info = sgetrf(handle, a)
    lu, wpiv, winfo = oracle.sgetrf_batched(a[None])
    assert st == aclsolver.SUCCESS
    assert info == winfo[0] == 201
    assert np.array_equal(ipiv, wpiv[0])
    assert same_bits(got, lu[0]), first_mismatch(got, lu[0])


def test_large_sgetrf_rejects_non_finite_input(handle):
    """As for every order: a NaN or Inf entry is refused before factoring (INVALID_VALUE,
    info -3) and A is left as it was."""
    n = 600
    a = gaussian(n, n, seed=4)
    a[450, 460] = np.nan
    st, got, _, info = sgetrf(handle, a)
    assert st == aclsolver.INVALID_VALUE and info == -3
    assert same_bits(got, a)


def test_large_sgetrf_without_pivoting(handle):
    n = 600
    a = gaussian(n, n, seed=3) + 40 * np.eye(n, dtype=np.float32)
    st, got, _, info = sgetrf(handle, a, pivoting=False)
    lu, _, winfo = oracle.sgetrf_batched(a[None], pivoting=False)
    assert st == aclsolver.SUCCESS and info == winfo[0] == 0
    assert same_bits(got, lu[0]), first_mismatch(got, lu[0])


def test_large_sgetrf_8192_backward_error(handle):
    """The full 8192 x 8192 order: every panel row of the cluster is occupied.  The factors
    must solve A x = b to FP32-level backward error (in FP64 arithmetic on the host)."""
    n = 8192
    a = gaussian(n, n, seed=6)
    st, got, ipiv, info = sgetrf(handle, a, pad=0)
    assert st == aclsolver.SUCCESS and info == 0
    assert np.all(ipiv >= np.arange(1, n + 1)) and np.all(ipiv <= n)
    b = np.random.default_rng(7).standard_normal(n)
    pb = b.copy()
    for k in range(n):
        r = ipiv[k] - 1
        if r != k:
            pb[[k, r]] = pb[[r, k]]
    lu = got.astype(np.float64)
    y = sla.solve_triangular(lu, pb, lower=True, unit_diagonal=True, check_finite=False)
    x = sla.solve_triangular(lu, y, lower=False, check_finite=False)
    a64 = a.astype(np.float64)
    berr = np.abs(b - a64 @ x).max() / (np.abs(a64).sum(axis=1).max() * np.abs(x).max() + np.abs(b).max())
    assert berr < 1e-6, berr


# ---- refinement of one large system (aclsolverSgesvIrBatched, batchSize 1, n > 512) ------

def gesv_ir_one(handle, a, b, precision, max_iter=10, tol=1e-7):
    lib = aclsolver.library()
    n = a.shape[0]
    nrhs = b.shape[1]
    da = DeviceMatrices(a[None], ld=n + 1)
    db = DeviceMatrices(b[None], ld=n + 2)
    dx = DeviceMatrices(np.zeros_like(b)[None], ld=n + 3)
    iters = torch.full((1,), -5, dtype=torch.int32, device="cuda")
    berr = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    info = info_buffer(1)
    st = lib.aclsolverSgesvIrBatched(handle.value, precision, n, nrhs, da.table_ptr, da.ld, db.table_ptr, db.ld,
                                    dx.table_ptr, dx.ld, max_iter, tol, iters.data_ptr(), berr.data_ptr(),
                                    info.data_ptr(), 1)
    handle.stream.synchronize()
    assert da.unchanged() and db.unchanged(), "A and B must be left as they were"
    return st, dx.read()[0], int(iters.cpu()[0]), float(berr.cpu()[0]), int(info.cpu()[0])


def test_large_ir_fp32_without_refinement(handle):
    """maxIter 0 in FP32: the whole-GPU factorisation (the oracle's factors) and one solve
    whose diagonal blocks go through their inverses (not the oracle's rounding order): an
    FP32-accurate solution whose reported backward error is its own."""
    n = 700
    a = gaussian(n, n, seed=21)
    b = np.random.default_rng(22).standard_normal((n, 3)).astype(np.float32)
    st, x, iters, berr, info = gesv_ir_one(handle, a, b, aclsolver.FACTOR_FP32, max_iter=0)
    assert st == aclsolver.SUCCESS and info == 0 and iters == 0
    lu, ipiv, _ = oracle.sgetrf_batched(a[None])
    want = oracle.sgetrs_batched(lu, ipiv, b[None])[0]
    assert np.max(np.abs(x - want)) <= 1e-3 * np.max(np.abs(want))
    be = max(judges.backward_error(a, x[:, j], b[:, j]) for j in range(3))
    assert be <= 1e-6
    assert berr == pytest.approx(be, rel=1e-6)


@pytest.mark.parametrize("precision", ["FACTOR_BF16X3", "FACTOR_FP32"])
@pytest.mark.parametrize("n,kappa", [(1000, 1e4), (2048, 1e3)])
def test_large_ir_reaches_fp32_backward_error(handle, precision, n, kappa):
    a = conditioned_batch(1, n, kappa, seed=n)[0]
    b = np.random.default_rng(n + 1).standard_normal((n, 4)).astype(np.float32)
    st, x, iters, berr, info = gesv_ir_one(handle, a, b, getattr(aclsolver, precision), max_iter=10, tol=1e-7)
    assert st == aclsolver.SUCCESS and info == 0
    for j in range(4):
        be = judges.backward_error(a, x[:, j], b[:, j])
        assert be <= 1e-6, (j, be, berr, iters)
        assert judges.forward_error(a, x[:, j], b[:, j]) <= kappa * 1e-6
    assert 0 <= iters <= 10 and berr <= 1e-6


def test_large_ir_singular_is_not_solved(handle):
    n = 600
    a = gaussian(n, n, seed=31)
    a[:, 100] = 0.0
    b = np.ones((n, 1), dtype=np.float32)
    st, x, iters, berr, info = gesv_ir_one(handle, a, b, aclsolver.FACTOR_BF16X3)
    assert st == aclsolver.SUCCESS and info == 101
    assert np.all(x == 0.0) and np.isnan(berr) and iters == 0


def test_large_ir_8192_split_bf16(handle):
    """The single large system of the benchmark family: 8192 x 8192, A = U diag(s) V^T with
    kappa = 1e3 (generated on the GPU), 16 right-hand sides, split-BF16 factorisation plus
    FP64 refinement to FP32-level backward error (checked in FP64 on the GPU)."""
    n, nrhs = 8192, 16
    g = torch.Generator(device="cuda").manual_seed(6)
    u, _ = torch.linalg.qr(torch.randn(n, n, device="cuda", dtype=torch.float64, generator=g))
    v, _ = torch.linalg.qr(torch.randn(n, n, device="cuda", dtype=torch.float64, generator=g))
    s = torch.logspace(0.0, -3.0, n, device="cuda", dtype=torch.float64)
    a64 = (u * s) @ v.T
    del u, v
    a = a64.float()
    b = torch.randn(n, nrhs, device="cuda", generator=g).float()
    lib = aclsolver.library()
    # column-major device buffers: the transposes of the row-major torch tensors
    at = a.T.contiguous()
    bt = b.T.contiguous()
    xt = torch.zeros_like(bt)
    tables = [aclsolver.pointer_table(t, 1, 0) for t in (at, bt, xt)]
    iters = torch.zeros(1, dtype=torch.int32, device="cuda")
    berr = torch.zeros(1, dtype=torch.float64, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = lib.aclsolverSgesvIrBatched(handle.value, aclsolver.FACTOR_BF16X3, n, nrhs, tables[0].data_ptr(), n,
                                    tables[1].data_ptr(), n, tables[2].data_ptr(), n, 10, 1e-7, iters.data_ptr(),
                                    berr.data_ptr(), info.data_ptr(), 1)
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS and int(info.item()) == 0
    x = xt.T.double()
    a32 = a.double()
    r = b.double() - a32 @ x
    be = (r.abs().amax(dim=0) / (a32.abs().sum(dim=1).max() * x.abs().amax(dim=0) + b.double().abs().amax(dim=0)))
    assert float(be.max()) <= 1e-6, (be.max(), berr, iters)
    assert 0 <= int(iters.item()) <= 10


@pytest.mark.parametrize("n,nrhs", [(700, 1), (1000, 16), (2048, 5)])
def test_large_sgetrs_one_system_matches_oracle(handle, n, nrhs):
    """aclsolverSgetrsBatched with one system above 512: the whole-GPU sweep, bit for bit."""
    lib = aclsolver.library()
    a = gaussian(n, n, seed=n + 40)
    lu, ipiv, _ = oracle.sgetrf_batched(a[None])
    b = np.random.default_rng(n + 41).standard_normal((n, nrhs)).astype(np.float32)
    da = DeviceMatrices(lu, ld=n + 1)
    db = DeviceMatrices(b[None], ld=n + 3)
    piv = device_ints(ipiv.reshape(-1))
    info = info_buffer(1)
    st = lib.aclsolverSgetrsBatched(handle.value, 0, n, nrhs, da.table_ptr, da.ld, piv.data_ptr(), db.table_ptr,
                                   db.ld, info.data_ptr(), 1)
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS and int(info.cpu()[0]) == 0
    want = oracle.sgetrs_batched(lu, ipiv, b[None])[0]
    got = db.read()[0]
    assert same_bits(got, want), first_mismatch(got, want)


@pytest.mark.parametrize("pattern", ["identity", "last_row", "adjacent", "chunk_edges", "random"])
def test_large_sgetrs_pivot_patterns(handle, pattern):
    """Pivot sequences that no factorisation of a random matrix produces -- every swap with the
    last row, a chain of adjacent swaps, swaps across the 32-swap chunks the composition works
    in -- through the one-system solve, bit for bit against the oracle's sequential swaps."""
    lib = aclsolver.library()
    n, nrhs = 1100, 3
    rng = np.random.default_rng(60)
    lu = np.tril(rng.standard_normal((n, n)), -1) * 0.05 + np.triu(rng.standard_normal((n, n)), 1) * 0.05
    lu[np.arange(n), np.arange(n)] = 2.0 + rng.random(n)
    lu = lu.astype(np.float32)[None]
    k = np.arange(n)
    if pattern == "identity":
        ipiv = k + 1
    elif pattern == "last_row":
        ipiv = np.full(n, n)
    elif pattern == "adjacent":
        ipiv = np.minimum(k + 2, n)
    elif pattern == "chunk_edges":
        ipiv = np.where(k % 32 == 31, np.minimum(k + 33, n), np.minimum(k + 32 - k % 32, n))
    else:
        ipiv = k + 1 + (rng.random(n) * (n - k)).astype(np.int64)
    ipiv = ipiv.astype(np.int32).reshape(1, n)
    b = rng.standard_normal((n, nrhs)).astype(np.float32)
    da = DeviceMatrices(lu, ld=n)
    db = DeviceMatrices(b[None], ld=n)
    piv = device_ints(ipiv.reshape(-1))
    info = info_buffer(1)
    st = lib.aclsolverSgetrsBatched(handle.value, 0, n, nrhs, da.table_ptr, da.ld, piv.data_ptr(), db.table_ptr,
                                   db.ld, info.data_ptr(), 1)
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS and int(info.cpu()[0]) == 0
    want = oracle.sgetrs_batched(lu, ipiv, b[None])[0]
    got = db.read()[0]
    assert same_bits(got, want), first_mismatch(got, want)


def test_large_sgetrs_bad_pivot_leaves_b(handle):
    lib = aclsolver.library()
    n = 640
    a = gaussian(n, n, seed=50)
    lu, ipiv, _ = oracle.sgetrf_batched(a[None])
    ipiv = ipiv.copy()
    ipiv[0, 300] = n + 5
    b = np.random.default_rng(51).standard_normal((n, 2)).astype(np.float32)
    da = DeviceMatrices(lu, ld=n)
    db = DeviceMatrices(b[None], ld=n)
    piv = device_ints(ipiv.reshape(-1))
    info = info_buffer(1)
    st = lib.aclsolverSgetrsBatched(handle.value, 0, n, 2, da.table_ptr, da.ld, piv.data_ptr(), db.table_ptr, db.ld,
                                   info.data_ptr(), 1)
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS and int(info.cpu()[0]) == -6
    assert np.array_equal(db.read()[0], b)
