"""aclsolverSgesvIrBatched on the GPU: LU in FP32, BF16 or split-BF16 precision plus FP64
iterative refinement, judged against an FP64 LAPACK solve (backward and forward error) and,
with no refinement in FP32 mode, against the oracle's sgetrf + sgetrs (bit for bit up to order 64)."""

import numpy as np
import pytest
import torch

import aclsolver
import oracle
from oracle import judges
from helpers import DeviceMatrices, conditioned_batch, first_mismatch, info_buffer, same_bits

pytestmark = pytest.mark.gpu


def gesv_ir(handle, a, b, precision, max_iter=10, tol=1e-7, x_init=None):
    lib = aclsolver.library()
    count, n, _ = a.shape
    nrhs = b.shape[2]
    da = DeviceMatrices(a, ld=n + 1)
    db = DeviceMatrices(b, ld=n + 2)
    dx = DeviceMatrices(np.zeros_like(b) if x_init is None else x_init, ld=n + 3)
    iters = torch.full((count,), -5, dtype=torch.int32, device="cuda")
    berr = torch.full((count,), -1.0, dtype=torch.float64, device="cuda")
    info = info_buffer(count)
    st = lib.aclsolverSgesvIrBatched(handle.value, precision, n, nrhs, da.table_ptr, da.ld, db.table_ptr, db.ld,
                                    dx.table_ptr, dx.ld, max_iter, tol, iters.data_ptr(), berr.data_ptr(),
                                    info.data_ptr(), count)
    handle.stream.synchronize()
    assert da.unchanged() and db.unchanged(), "A and B must be left as they were"
    return st, dx.read(), iters.cpu().numpy(), berr.cpu().numpy(), info.cpu().numpy()


def rhs(count, n, nrhs, seed):
    return np.random.default_rng(seed).standard_normal((count, n, nrhs)).astype(np.float32)


@pytest.mark.parametrize("n", [40, 100, 129, 333, 512])
def test_fp32_without_refinement_is_sgetrf_sgetrs(handle, n):
    """maxIter 0 in FP32: the oracle's sgetrf + sgetrs (bit for bit up to order 64)."""
    a = np.random.default_rng(n).standard_normal((3, n, n)).astype(np.float32)
    b = rhs(3, n, 2, n + 1)
    st, x, iters, berr, info = gesv_ir(handle, a, b, aclsolver.FACTOR_FP32, max_iter=0)
    assert st == aclsolver.SUCCESS and np.all(info == 0) and np.all(iters == 0)
    lu, ipiv, _ = oracle.sgetrf_batched(a)
    want = oracle.sgetrs_batched(lu, ipiv, b)
    if n <= 64:
        assert same_bits(x, want), first_mismatch(x, want)
    else:
        # above 64 the solves apply the diagonal 32 x 32 triangles through their inverses
        # (a different rounding order than sgetrs): the same factors, an FP32-accurate solve
        for q in range(3):
            for j in range(2):
                assert judges.backward_error(a[q], x[q][:, j], b[q][:, j]) <= 1e-6
        assert np.max(np.abs(x - want)) <= 1e-3 * np.max(np.abs(want))
    for q in range(3):  # the reported berr is that of the (FP64) iterate, i.e. of x here
        want = max(judges.backward_error(a[q], x[q][:, j], b[q][:, j]) for j in range(2))
        assert berr[q] == pytest.approx(want, rel=1e-6)


@pytest.mark.parametrize("precision", ["FACTOR_FP32", "FACTOR_BF16X3"])
@pytest.mark.parametrize("kappa", [1e2, 1e4, 1e5])
def test_refinement_reaches_fp32_backward_error(handle, precision, kappa):
    n, count = 256, 4
    a = conditioned_batch(count, n, kappa, seed=int(np.log10(kappa)))
    b = rhs(count, n, 1, 9)
    st, x, iters, berr, info = gesv_ir(handle, a, b, getattr(aclsolver, precision), max_iter=10, tol=1e-7)
    assert st == aclsolver.SUCCESS and np.all(info == 0)
    for q in range(count):
        be = judges.backward_error(a[q], x[q], b[q])
        fe = judges.forward_error(a[q], x[q], b[q])
        assert be <= 1e-6, (q, be, berr[q], iters[q])
        # the reported error is that of the FP64 iterate; x is its FP32 rounding, so the two
        # agree to within the rounding's share (a zero or stale report fails here)
        assert 0.0 < berr[q] <= 1e-6
        assert berr[q] <= 2.0 * be + 1e-7 and be <= 2.0 * berr[q] + 1e-7, (q, be, berr[q])
        assert fe <= kappa * 1e-6, (q, fe)
        assert 0 <= iters[q] <= 10


def test_bf16_refinement_well_conditioned(handle):
    """Plain BF16 trailing updates (unit roundoff 2^-8) still refine to FP32 backward error
    when kappa * u stays well below one."""
    n, count = 200, 3
    a = conditioned_batch(count, n, 10.0, seed=21)
    b = rhs(count, n, 3, 22)
    st, x, iters, berr, info = gesv_ir(handle, a, b, aclsolver.FACTOR_BF16, max_iter=30, tol=1e-7)
    assert st == aclsolver.SUCCESS and np.all(info == 0)
    for q in range(count):
        assert judges.backward_error(a[q], x[q], b[q]) <= 1e-6
        assert iters[q] >= 1  # BF16 factors alone are far from FP32 accuracy


def test_bf16_reports_honest_error_when_it_cannot_converge(handle):
    """At kappa = 1e5 BF16 LU is too inaccurate for classic refinement: the call must stop
    (stall rule) and report a backward error that matches the returned solution."""
    n, count = 256, 2
    a = conditioned_batch(count, n, 1e5, seed=5)
    b = rhs(count, n, 1, 6)
    st, x, iters, berr, info = gesv_ir(handle, a, b, aclsolver.FACTOR_BF16, max_iter=10, tol=1e-7)
    assert st == aclsolver.SUCCESS and np.all(info == 0)
    for q in range(count):
        be = judges.backward_error(a[q], x[q], b[q])
        assert np.isfinite(berr[q])
        # berr is that of the FP64 iterate; X is its FP32 rounding (relative 6e-8 per entry)
        assert abs(be - berr[q]) <= 1e-7 + 0.05 * berr[q]


@pytest.mark.parametrize("n, nrhs", [(257, 9), (333, 3), (130, 17)])
def test_ragged_orders_and_rhs_groups(handle, n, nrhs):
    """Orders with a partial last panel and outer block, and right-hand sides spread over
    several solve blocks: the refinement's solves apply the panels' row changes block by
    block (no left interchanges) and must match the LAPACK-form solve's accuracy."""
    count = 4
    a = conditioned_batch(count, n, 1e4, seed=n)
    b = rhs(count, n, nrhs, n + 7)
    st, x, iters, berr, info = gesv_ir(handle, a, b, aclsolver.FACTOR_FP32, max_iter=0)
    assert st == aclsolver.SUCCESS and np.all(info == 0)
    lu, ipiv, _ = oracle.sgetrf_batched(a)
    want = oracle.sgetrs_batched(lu, ipiv, b)
    assert np.max(np.abs(x - want)) <= 1e-3 * np.max(np.abs(want))
    st, x, iters, berr, info = gesv_ir(handle, a, b, aclsolver.FACTOR_BF16X3, max_iter=5, tol=1e-7)
    assert st == aclsolver.SUCCESS and np.all(info == 0)
    for q in range(count):
        for j in range(nrhs):
            assert judges.backward_error(a[q], x[q][:, j], b[q][:, j]) <= 1e-6, (q, j)


def test_small_orders_and_several_rhs(handle):
    n, count = 48, 5
    a = conditioned_batch(count, n, 1e3, seed=2)
    b = rhs(count, n, 4, 3)
    st, x, iters, berr, info = gesv_ir(handle, a, b, aclsolver.FACTOR_BF16X3, max_iter=5, tol=1e-7)
    assert st == aclsolver.SUCCESS and np.all(info == 0)
    for q in range(count):
        assert judges.backward_error(a[q], x[q], b[q]) <= 1e-6


def test_singular_matrix_is_not_solved(handle):
    n = 90
    a = conditioned_batch(3, n, 10.0, seed=4)
    a[1, :, 7] = 0.0
    b = rhs(3, n, 1, 5)
    x0 = np.full_like(b, 2.5)
    st, x, iters, berr, info = gesv_ir(handle, a, b, aclsolver.FACTOR_BF16X3, x_init=x0)
    assert st == aclsolver.SUCCESS
    assert info[0] == 0 and info[1] > 0 and info[2] == 0
    assert np.all(x[1] == 2.5)
    assert np.isnan(berr[1]) and iters[1] == 0
    assert judges.backward_error(a[2], x[2], b[2]) <= 1e-6


def test_solution_may_overwrite_b(handle):
    lib = aclsolver.library()
    n, count = 130, 2
    a = conditioned_batch(count, n, 100.0, seed=8)
    b = rhs(count, n, 1, 9)
    da = DeviceMatrices(a, ld=n)
    db = DeviceMatrices(b, ld=n)
    info = info_buffer(count)
    st = lib.aclsolverSgesvIrBatched(handle.value, aclsolver.FACTOR_BF16X3, n, 1, da.table_ptr, n, db.table_ptr, n,
                                    db.table_ptr, n, 10, 1e-7, None, None, info.data_ptr(), count)
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS
    x = db.read()
    for q in range(count):
        assert judges.backward_error(a[q], x[q], b[q]) <= 1e-6


@pytest.mark.parametrize(
    "field,value,arg",
    [("precision", 2, 1), ("n", 8193, 2), ("nrhs", -1, 3), ("lda", 5, 5), ("ldb", 5, 7), ("ldx", 5, 9),
     ("max_iter", -1, 10), ("tol", -1.0, 11), ("batch", -1, 15)],
)
def test_argument_errors(handle, field, value, arg):
    lib = aclsolver.library()
    n, count = 16, 2
    a = conditioned_batch(count, n, 10.0, seed=1)
    da = DeviceMatrices(a, ld=n)
    db = DeviceMatrices(rhs(count, n, 1, 2), ld=n)
    dx = DeviceMatrices(rhs(count, n, 1, 3), ld=n)
    args = dict(precision=aclsolver.FACTOR_FP32, n=n, nrhs=1, lda=n, ldb=n, ldx=n, max_iter=3, tol=1e-7, batch=count)
    args[field] = value
    info = info_buffer(count)
    st = lib.aclsolverSgesvIrBatched(handle.value, args["precision"], args["n"], args["nrhs"], da.table_ptr,
                                    args["lda"], db.table_ptr, args["ldb"], dx.table_ptr, args["ldx"],
                                    args["max_iter"], args["tol"], None, None, info.data_ptr(), args["batch"])
    handle.stream.synchronize()
    assert st == aclsolver.INVALID_VALUE
    got = info.cpu().numpy()
    assert got[0] == -arg


def lu_reconstruction_error(a, got, ipiv):
    """max |L U - P A| / max |A| in FP64 for packed factors and LAPACK pivots."""
    n = a.shape[0]
    L = np.tril(got.astype(np.float64), -1) + np.eye(n)
    U = np.triu(got.astype(np.float64))
    pa = a.astype(np.float64).copy()
    for k in range(n):
        r = ipiv[k] - 1
        if r != k:
            pa[[k, r]] = pa[[r, k]]
    return np.abs(L @ U - pa).max() / np.abs(a).max()


@pytest.mark.parametrize("n", [96, 129, 200, 300, 512])
def test_sgetrf_batched_mixed(handle, n):
    """FP32 precision is aclsolverSgetrfBatched bit for bit; the split-BF16 factors reproduce
    P A = L U to about FP32 accuracy, the BF16 ones to about BF16 accuracy (the outer blocks'
    U12 go through the inverse of their L11 on the tensor cores in both)."""
    lib = aclsolver.library()
    a = conditioned_batch(3, n, 1e3, seed=n)
    a[2, :, 70] = 0.0  # a zero pivot: info 71, the column takes no part in later updates
    lu, wpiv, winfo = oracle.sgetrf_batched(a)
    assert winfo.tolist() == [0, 0, 71]
    bounds = {aclsolver.FACTOR_BF16X3: 3e-4, aclsolver.FACTOR_BF16: 0.25}
    for precision in (aclsolver.FACTOR_FP32, aclsolver.FACTOR_BF16X3, aclsolver.FACTOR_BF16):
        dm = DeviceMatrices(a, ld=n + 2)
        piv = torch.zeros(3 * n, dtype=torch.int32, device="cuda")
        info = info_buffer(3)
        st = lib.aclsolverSgetrfBatchedMixed(handle.value, precision, n, dm.table_ptr, dm.ld, piv.data_ptr(),
                                            info.data_ptr(), 3)
        handle.stream.synchronize()
        assert st == aclsolver.SUCCESS and info.cpu().tolist() == [0, 0, 71]
        got = dm.read()
        ipiv = piv.cpu().numpy().reshape(3, n)
        if precision == aclsolver.FACTOR_FP32:
            assert np.array_equal(ipiv, wpiv)
            assert same_bits(got, lu), first_mismatch(got, lu)
        else:
            for q in range(3):
                rel = lu_reconstruction_error(a[q], got[q], ipiv[q])
                assert rel < bounds[precision], (precision, q, rel)
