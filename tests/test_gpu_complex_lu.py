"""The complex LU family on the GPU through the C ABI: Cgetrf, Cgetrs (host buffers), Cgetri,
CgetriBatched and CmatinvBatched, each bit for bit the oracle's restatement (oracle.c,
orc_cgetrf / orc_cgetrs / orc_cgetri / orc_cmatinv), with the reference's own acceptance
gates on its data recipes (test/cgetrf/data/verify_result.py, test/utils/lu_verify_utils.py,
test/utils/verify_utils.py, test/cgetri_batched/data/verify_result.py)."""

import ctypes

import numpy as np
import pytest
import torch

import aclsolver
import oracle
from oracle import judges
from helpers import info_buffer
from test_gpu_complex import CMatrices, cbits

pytestmark = pytest.mark.gpu


def crandn(rng, *shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)


def dominant(rng, count, n):
    """The reference's inverse recipe: N(0,1) parts, the diagonal raised to (row L1 + U(0,10)) (1+i)."""
    a = crandn(rng, count, n, n)
    for q in range(count):
        for i in range(n):
            s = np.sum(np.abs(a[q, i, :])) - np.abs(a[q, i, i])
            a[q, i, i] = (s + rng.random() * 10) * (1 + 1j)
    return a


def cgetrf(handle, a, pad=0, pivoting=True):
    lib = aclsolver.library()
    m, n = a.shape
    dm = CMatrices(a[None], m + pad)
    ipiv = info_buffer(max(1, min(m, n)))
    info = info_buffer(1)
    st = lib.aclsolverCgetrf(handle.value, m, n, dm.tensor.data_ptr(), dm.ld, None,
                             ipiv.data_ptr() if pivoting else None, info.data_ptr())
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS
    return dm.read()[0], ipiv.cpu().numpy()[: min(m, n)], int(info.cpu()[0])


def check_getrf(handle, a, pad=1, pivoting=True):
    got, piv, info = cgetrf(handle, a, pad, pivoting)
    want, wpiv, winfo = oracle.cgetrf_batched(a[None], pivoting=pivoting)
    assert info == winfo[0]
    if pivoting:
        assert np.array_equal(piv, wpiv[0])
    assert cbits(got, want[0])
    return got, piv, info


@pytest.mark.parametrize("m,n", [(1, 1), (2, 1), (1, 3), (5, 5), (32, 32), (33, 17), (17, 70), (100, 100),
                                 (150, 150), (200, 200), (300, 257), (257, 300), (800, 40), (20, 2000),
                                 (1000, 1000), (4096, 64), (2500, 700)])
def test_cgetrf_matches_oracle(handle, m, n):
    a = crandn(np.random.default_rng(m * 7 + n), m, n)
    check_getrf(handle, a, pad=3)


@pytest.mark.parametrize("m,n", [(64, 64), (512, 512)])
def test_cgetrf_reference_recipe_passes_its_gate(handle, m, n):
    """test/cgetrf/data/gen_data.py: integer parts 1..10 (m x 2n floats read as m x n complex);
    verify_result.py: |A - P^T L U| / |A| <= 1e-3 on all but 1e-4 of the entries."""
    rng = np.random.RandomState(149)
    a = rng.randint(1, 11, size=(m, n * 2)).astype(np.float32).view(np.complex64)
    got, piv, info = check_getrf(handle, a)
    assert info == 0
    assert judges.cgetrf_gate(a, got, piv)


def test_cgetrf_without_pivoting(handle):
    a = dominant(np.random.default_rng(5), 1, 90)[0]
    check_getrf(handle, a, pivoting=False)


def test_cgetrf_zero_column_sets_info(handle):
    a = crandn(np.random.default_rng(9), 120, 120)
    a[:, 37] = 0
    _, _, info = check_getrf(handle, a)
    assert info == 38


def test_cgetrf_extreme_scales_take_the_scaled_quotient(handle):
    """Entries whose exponents span 1e-38..1e38 drive Divide through its exponent-aligned
    branch (NeedsScaledNumerator); a column of one dominant pivot over 2000 rows gives 1999
    plain divisions each."""
    rng = np.random.default_rng(11)
    m = 2000
    e = rng.uniform(-37, 37, size=(m, 2))
    a = (rng.standard_normal(m) * 10.0 ** e[:, 0] + 1j * rng.standard_normal(m) * 10.0 ** e[:, 1]).astype(np.complex64)
    a[0] = np.complex64(3e38 + 2e38j)
    check_getrf(handle, a[:, None])
    for scale in (1e-30, 1e-12, 1e20):
        b = (crandn(rng, 64, 64) * np.float32(scale)).astype(np.complex64)
        b[rng.random((64, 64)) < 0.2] *= np.float32(1e-20)
        check_getrf(handle, b)


def test_cgetrf_nonfinite_entries(handle):
    a = crandn(np.random.default_rng(2), 50, 50)
    a[3, 4] = np.nan
    a[10, 1] = np.inf
    check_getrf(handle, a)


def test_cgetrf_order_4096_bits_and_gate(handle):
    """The largest order, blocked over the whole GPU: the oracle's bits and the reference gate."""
    rng = np.random.RandomState(149)
    a = rng.randint(1, 11, size=(4096, 8192)).astype(np.float32).view(np.complex64)
    got, piv, info = check_getrf(handle, a, pad=0)
    assert info == 0 and judges.cgetrf_gate(a, got, piv)


# ---- Cgetrs: host row-major buffers -------------------------------------------------------

def cgetrs(handle, trans, lu, piv, b, pad_a=0, pad_b=0):
    lib = aclsolver.library()
    n, nrhs = b.shape
    lda, ldb = n + pad_a, nrhs + pad_b
    ha = np.full((n, lda), np.complex64(7 + 7j), dtype=np.complex64)
    ha[:, :n] = lu  # row-major A(r, c) = ha[r, c]
    hb = np.full((n, ldb), np.complex64(9 + 9j), dtype=np.complex64)
    hb[:, :nrhs] = b
    hp = np.ascontiguousarray(piv, dtype=np.int32)
    info = np.array([-99], dtype=np.int32)
    st = lib.aclsolverCgetrs(handle.value, trans, n, nrhs, ha.ctypes.data, lda, hp.ctypes.data, hb.ctypes.data, ldb,
                             info.ctypes.data)
    assert st == 0 and info[0] == 0
    assert np.all(hb[:, nrhs:] == np.complex64(9 + 9j))
    return hb[:, :nrhs]


@pytest.mark.parametrize("trans", [0, 1, 2])
@pytest.mark.parametrize("n,nrhs", [(1, 1), (7, 3), (32, 32), (33, 5), (100, 40), (500, 17)])
def test_cgetrs_matches_oracle(handle, trans, n, nrhs):
    rng = np.random.default_rng(n * 3 + nrhs + trans)
    a = crandn(rng, 1, n, n)
    lu, piv, _ = oracle.cgetrf_batched(a)
    b = crandn(rng, 1, n, nrhs)
    got = cgetrs(handle, trans, lu[0], piv[0], b[0], pad_a=2, pad_b=1)
    want = oracle.cgetrs_batched(lu, piv, b, trans=trans)[0]
    assert cbits(got, want)


@pytest.mark.parametrize("trans", [0, 1, 2])
def test_cgetrs_reference_recipe_passes_its_gate(handle, trans):
    """test/cgetrs/data/gen_data.py recipe (integer parts 1..10, a dominant shuffled diagonal,
    scipy LU) compared like compare_and_report: |err| > 1e-3 and relative > 1e-3 on at most
    1e-4 of the entries."""
    import scipy.linalg

    n, nrhs = 256, 32
    rng = np.random.RandomState(149)
    a = (rng.randint(1, 11, size=(n, n)) + 1j * rng.randint(1, 11, size=(n, n))).astype(np.complex64)
    for i in range(n):
        s = np.sum(np.abs(a[i, :])) - np.abs(a[i, i])
        a[i, i] = s + rng.rand() * 10 + 1j * rng.rand() * 10
    rng.shuffle(a)
    b = (rng.randn(n, nrhs) + 1j * rng.randn(n, nrhs)).astype(np.complex64)
    lu, piv = scipy.linalg.lu_factor(a)
    lu = lu.astype(np.complex64)
    got = cgetrs(handle, trans, lu, piv + 1, b)
    want = scipy.linalg.lu_solve((lu, piv), b, trans=trans)
    assert judges.complex_solve_compare_ok(got, want)
    assert cbits(got, oracle.cgetrs_batched(lu[None], (piv + 1)[None], b[None], trans=trans)[0])


# ---- inverses -------------------------------------------------------------------------------

def getri_batched(handle, lu, piv, pad=1, with_pivots=True):
    lib = aclsolver.library()
    count, n, _ = lu.shape
    da = CMatrices(lu, n + pad)
    dc = CMatrices(np.zeros_like(lu), n + 2)
    dp = torch.tensor(np.ascontiguousarray(piv, dtype=np.int32).reshape(-1), device="cuda")
    info = info_buffer(count)
    st = lib.aclsolverCgetriBatched(handle.value, n, da.table.data_ptr(), da.ld,
                                    dp.data_ptr() if with_pivots else None, dc.table.data_ptr(), dc.ld,
                                    info.data_ptr(), count)
    handle.stream.synchronize()
    return st, dc, info.cpu().numpy()


@pytest.mark.parametrize("n", [1, 2, 5, 31, 32, 33, 64, 65, 100, 128, 129, 200, 256, 257, 300])
def test_cgetri_batched_matches_oracle(handle, n):
    rng = np.random.default_rng(n)
    count = 5 if n <= 256 else 2
    a = crandn(rng, count, n, n)
    lu, piv, _ = oracle.cgetrf_batched(a)
    st, dc, info = getri_batched(handle, lu, piv)
    want, winfo = oracle.cgetri_batched(lu, piv)
    assert st == aclsolver.SUCCESS and np.array_equal(info, winfo) and np.all(info == 0)
    assert cbits(dc.read(), want)


def test_cgetri_batched_singular_and_null_pivots(handle):
    rng = np.random.default_rng(3)
    n = 48
    a = dominant(rng, 6, n)
    lu, _, _ = oracle.cgetrf_batched(a, pivoting=False)
    lu[2, 17, 17] = 0  # zero diagonal: info 18, output unwritten
    piv = np.tile(np.arange(1, n + 1, dtype=np.int32), (6, 1))
    st, dc, info = getri_batched(handle, lu, piv, with_pivots=False)
    want, winfo = oracle.cgetri_batched(lu, None)
    assert st == aclsolver.SUCCESS and info.tolist() == winfo.tolist() and info[2] == 18
    out = dc.read()
    ok = [q for q in range(6) if q != 2]
    assert cbits(out[ok], want[ok])
    assert np.all(out[2] == 0), "a failed matrix's output must stay unwritten"


def test_cgetri_batched_bad_pivot_reports_minus_four(handle):
    n = 20
    a = crandn(np.random.default_rng(4), 3, n, n)
    lu, piv, _ = oracle.cgetrf_batched(a)
    piv = piv.copy()
    piv[1, 5] = 3  # below its row: invalid
    st, _, info = getri_batched(handle, lu, piv)
    assert st == aclsolver.INVALID_VALUE and info[1] == -4 and info[0] == 0 and info[2] == 0


def test_cgetri_reference_recipe_passes_its_gate(handle):
    """test/cgetri_batched/data/gen_data.py recipe: outputs within isclose(5e-3, 5e-3) of
    numpy's inverse on all but 1e-4 of the entries."""
    n, count = 48, 4
    np.random.seed(42)
    a = (np.random.randn(count, n, n).astype(np.float32) + 1j * np.random.randn(count, n, n).astype(np.float32))
    for b in range(count):
        for i in range(n):
            s = np.sum(np.abs(a[b, i, :])) - np.abs(a[b, i, i])
            a[b, i, i] = (s + np.random.rand() * 10) * (1 + 1j)
    a = a.astype(np.complex64)
    lu, piv, _ = oracle.cgetrf_batched(a)
    st, dc, info = getri_batched(handle, lu, piv)
    assert st == aclsolver.SUCCESS and np.all(info == 0)
    out = dc.read()
    for q in range(count):
        assert judges.inverse_golden_ok(out[q], np.linalg.inv(a[q]).astype(np.complex64))


@pytest.mark.parametrize("n", [16, 100, 256, 300, 600])
def test_cgetri_in_place(handle, n):
    lib = aclsolver.library()
    rng = np.random.default_rng(n + 1)
    a = crandn(rng, 1, n, n)
    lu, piv, _ = oracle.cgetrf_batched(a)
    da = CMatrices(lu, n + 3)
    lwork = ctypes.c_int(-1)
    assert lib.aclsolverCgetri_bufferSize(handle.value, n, da.tensor.data_ptr(), da.ld,
                                          ctypes.byref(lwork)) == aclsolver.SUCCESS
    assert lwork.value == n * n
    work = torch.zeros(2 * n * n, dtype=torch.float32, device="cuda")
    dp = torch.tensor(piv.reshape(-1), device="cuda")
    info = info_buffer(1)
    st = lib.aclsolverCgetri(handle.value, n, da.tensor.data_ptr(), da.ld, dp.data_ptr(), work.data_ptr(),
                             lwork.value, info.data_ptr())
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS and int(info.cpu()[0]) == 0
    want, _ = oracle.cgetri_batched(lu, piv)
    got = da.read()
    assert cbits(got, want)
    assert judges.inverse_judge(a[0], got[0])[0]


def matinv(handle, a, pad=0):
    lib = aclsolver.library()
    count, n, _ = a.shape
    da = CMatrices(a, n + pad)
    dc = CMatrices(np.zeros_like(a), n + 1)
    info = info_buffer(count)
    st = lib.aclsolverCmatinvBatched(handle.value, n, da.table.data_ptr(), da.ld, dc.table.data_ptr(), dc.ld,
                                     info.data_ptr(), count)
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS
    return dc.read(), info.cpu().numpy()


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 8, 9, 16, 17, 24, 31, 32])
def test_cmatinv_batched_matches_oracle(handle, n):
    rng = np.random.default_rng(100 + n)
    a = crandn(rng, 300, n, n)
    got, info = matinv(handle, a, pad=2)
    want, winfo = oracle.cmatinv_batched(a)
    assert np.array_equal(info, winfo) and np.all(info == 0)
    assert cbits(got, want)


def test_cmatinv_batched_singular_leaves_output(handle):
    rng = np.random.default_rng(7)
    n = 12
    a = crandn(rng, 10, n, n)
    a[4, :, 3] = 0
    a[7] = 0
    got, info = matinv(handle, a)
    want, winfo = oracle.cmatinv_batched(a)
    assert info.tolist() == winfo.tolist() and info[4] > 0 and info[7] == 1
    ok = [q for q in range(10) if info[q] == 0]
    assert cbits(got[ok], want[ok])
    assert np.all(got[4] == 0) and np.all(got[7] == 0)


def test_cmatinv_reference_recipe_passes_its_gate(handle):
    """test/cmatinv_batched/data/gen_data.py recipe (n = 3 default and the 32 bound)."""
    for n in (3, 32):
        np.random.seed(42)
        count = 64
        a = (np.random.randn(count, n, n).astype(np.float32) + 1j * np.random.randn(count, n, n).astype(np.float32))
        for b in range(count):
            for i in range(n):
                s = np.sum(np.abs(a[b, i, :])) - np.abs(a[b, i, i])
                a[b, i, i] = (s + np.random.rand() * 10) * (1 + 1j)
        a = a.astype(np.complex64)
        got, info = matinv(handle, a)
        assert np.all(info == 0)
        for q in range(count):
            assert judges.inverse_golden_ok(got[q], np.linalg.inv(a[q]).astype(np.complex64))
