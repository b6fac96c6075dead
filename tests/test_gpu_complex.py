"""Complex64 Cholesky parity through the C ABI on the GPU: CpotrfBatched, CpotrsBatched
(+ the multi-RHS addition), Cpotrf, Cpotrs -- bitwise against the oracle's order, within
1e-5 relative of FP64 LAPACK, and inside the reference's complex128 residual gate."""

import ctypes as C

import numpy as np
import pytest
import scipy.linalg as la

import aclsolver
import oracle
from oracle import judges
from helpers import info_buffer, same_bits

pytestmark = pytest.mark.gpu
SENTINEL = np.complex64(93 - 47j)  # the reference fixtures' padding value
SIZES = [1, 2, 7, 8, 9, 16, 17, 31, 32, 33, 48, 64, 65, 100, 128, 129, 160, 200, 240]


def hpd(count, n, seed):
    """A = G G^H / n + I, G real and imaginary parts N(0,1) (the uneven-batch recipe)."""
    rng = np.random.default_rng(seed)
    g = rng.standard_normal((count, n, n)) + 1j * rng.standard_normal((count, n, n))
    return (g @ g.conj().transpose(0, 2, 1) / n + np.eye(n)).astype(np.complex64)


class CMatrices:
    def __init__(self, mats, ld):
        import torch

        mats = np.asarray(mats, dtype=np.complex64)
        self.count, self.rows, self.cols = mats.shape
        self.ld = ld
        storage = np.full((self.count, self.cols, ld), SENTINEL, dtype=np.complex64)
        storage[:, :, : self.rows] = mats.transpose(0, 2, 1)
        self.initial = storage.copy()
        self.tensor = torch.from_numpy(storage.view(np.float32).reshape(-1)).cuda()
        self.table = aclsolver.pointer_table(self.tensor, self.count, self.cols * ld * 8)

    def raw(self):
        return self.tensor.cpu().numpy().view(np.complex64).reshape(self.count, self.cols, self.ld)

    def read(self):
        raw = self.raw()
        assert np.all(raw[:, :, self.rows :] == SENTINEL), "padding overwritten"
        return np.ascontiguousarray(raw[:, :, : self.rows].transpose(0, 2, 1))

    def unchanged(self):
        return np.array_equal(self.raw().view(np.uint32), self.initial.view(np.uint32))


def cbits(a, b):
    return same_bits(np.asarray(a).view(np.float32), np.asarray(b).view(np.float32))


def factor_batched(handle, a, upper, pad=2):
    lib = aclsolver.library()
    count, n, _ = a.shape
    dm = CMatrices(a, n + pad)
    info = info_buffer(count)
    st = lib.aclsolverCpotrfBatched(handle.value, int(upper), n, dm.table.data_ptr(), dm.ld, info.data_ptr(), count)
    handle.stream.synchronize()
    return st, dm, info.cpu().numpy()


@pytest.mark.parametrize("upper", [False, True])
@pytest.mark.parametrize("n", SIZES)
def test_cpotrf_batched(handle, n, upper):
    a = hpd(5, n, seed=n)
    st, dm, info = factor_batched(handle, a, upper)
    assert st == aclsolver.SUCCESS and np.all(info == 0)
    got = dm.read()
    want, _ = oracle.cpotrf_batched(a, upper=upper)
    assert cbits(got, want)
    ratios, cpu = [], []
    for q in range(len(a)):
        tri = np.triu(got[q]) if upper else np.tril(got[q])
        a64 = a[q].astype(np.complex128)
        gold = la.cholesky(a64, lower=not upper)
        assert np.abs(tri - gold).max() <= 1e-5 * max(1.0, np.abs(gold).max())
        full = np.triu(a[q]) + np.triu(a[q], 1).conj().T if upper else np.tril(a[q]) + np.tril(a[q], -1).conj().T
        ratios.append(judges.complex_ratio("potrf", full, got[q], upper))
        cpu.append(judges.complex_cpu_ratio("potrf", full, upper))
    assert not judges.residual_gate(ratios, cpu), judges.residual_gate(ratios, cpu)


def test_cpotrf_batched_failures_and_null_slot(handle):
    lib = aclsolver.library()
    n = 20
    a = hpd(4, n, seed=3)
    a[1, 7, 7] = -1.0
    a[2, 12, 12] = np.nan
    dm = CMatrices(a, n)
    dm.table[3] = 0
    info = info_buffer(4)
    st = lib.aclsolverCpotrfBatched(handle.value, 0, n, dm.table.data_ptr(), n, info.data_ptr(), 4)
    handle.stream.synchronize()
    want, winfo = oracle.cpotrf_batched(a[:3])
    assert st == aclsolver.SUCCESS
    assert info.cpu().tolist() == [0, int(winfo[1]), int(winfo[2]), -3]
    assert cbits(dm.read()[:3], want)


@pytest.mark.parametrize("args,code", [((2, 4, True, 4), -1), ((0, -1, True, 4), -2), ((0, 4, False, 4), -3),
                                       ((0, 4, True, 3), -4)])
def test_cpotrf_batched_argument_errors_write_first_slot(handle, args, code):
    lib = aclsolver.library()
    uplo, n, table, lda = args
    dm = CMatrices(hpd(2, 4, seed=1), 4)
    info = info_buffer(2)
    st = lib.aclsolverCpotrfBatched(handle.value, uplo, n, dm.table.data_ptr() if table else None, lda,
                                   info.data_ptr(), 2)
    handle.stream.synchronize()
    assert st == aclsolver.INVALID_VALUE
    assert info.cpu().tolist()[0] == code


def test_complex_null_handle_is_not_initialized(handle):
    lib = aclsolver.library()
    info = info_buffer(1)
    assert lib.aclsolverCpotrfBatched(None, 0, 4, None, 4, info.data_ptr(), 1) == aclsolver.NOT_INITIALIZED


@pytest.mark.parametrize("upper", [False, True])
@pytest.mark.parametrize("n", [1, 8, 17, 32, 33, 64, 100, 128, 150, 240, 241])
def test_cpotrs_batched(handle, n, upper):
    lib = aclsolver.library()
    a = hpd(4, n, seed=100 + n)
    f, _ = oracle.cpotrf_batched(a, upper=upper)
    rng = np.random.default_rng(n)
    b = (rng.standard_normal((4, n, 1)) + 1j * rng.standard_normal((4, n, 1))).astype(np.complex64)
    da, db = CMatrices(f, n + 1), CMatrices(b, n + 3)
    info = info_buffer(1)
    st = lib.aclsolverCpotrsBatched(handle.value, int(upper), n, 1, da.table.data_ptr(), da.ld, db.table.data_ptr(),
                                   db.ld, info.data_ptr(), 4)
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS and int(info.cpu()[0]) == 0
    assert da.unchanged()
    want = oracle.cpotrs_batched(f, b, upper=upper)
    assert cbits(db.read(), want)
    ratios, cpu = [], []
    for q in range(4):
        full = np.tril(a[q]) + np.tril(a[q], -1).conj().T if not upper else np.triu(a[q]) + np.triu(a[q], 1).conj().T
        ratios.append(judges.complex_ratio("potrs", full, db.read()[q], upper, b[q]))
        cpu.append(judges.complex_cpu_ratio("potrs", full, upper, b[q]))
    assert not judges.residual_gate(ratios, cpu), judges.residual_gate(ratios, cpu)


def test_cpotrs_batched_requires_single_rhs_and_multi_rhs_addition(handle):
    lib = aclsolver.library()
    n, nrhs = 24, 4
    a = hpd(3, n, seed=9)
    f, _ = oracle.cpotrf_batched(a)
    rng = np.random.default_rng(1)
    b = (rng.standard_normal((3, n, nrhs)) + 1j * rng.standard_normal((3, n, nrhs))).astype(np.complex64)
    da, db = CMatrices(f, n), CMatrices(b, n)
    info = info_buffer(1)
    st = lib.aclsolverCpotrsBatched(handle.value, 0, n, nrhs, da.table.data_ptr(), n, db.table.data_ptr(), n,
                                   info.data_ptr(), 3)
    handle.stream.synchronize()
    assert st == aclsolver.INVALID_VALUE and int(info.cpu()[0]) == -3
    st = lib.aclsolverCpotrsBatchedMultiRhs(handle.value, 0, n, nrhs, da.table.data_ptr(), n, db.table.data_ptr(),
                                           n, info.data_ptr(), 3)
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS and int(info.cpu()[0]) == 0
    assert cbits(db.read(), oracle.cpotrs_batched(f, b))


@pytest.mark.parametrize("n,nrhs", [(1, 1), (5, 3), (32, 2), (65, 4), (200, 2)])
def test_cpotrf_cpotrs_single(handle, n, nrhs):
    lib = aclsolver.library()
    a = hpd(1, n, seed=n)
    da = CMatrices(a, n + 1)
    lw = C.c_int(-1)
    assert lib.aclsolverCpotrf_bufferSize(handle.value, 0, n, da.tensor.data_ptr(), da.ld, C.byref(lw)) == 0
    info = info_buffer(1)
    st = lib.aclsolverCpotrf(handle.value, 0, n, da.tensor.data_ptr(), da.ld, None, 0, info.data_ptr())
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS and int(info.cpu()[0]) == 0
    want, _ = oracle.cpotrf_batched(a)
    assert cbits(da.read(), want)
    rng = np.random.default_rng(n)
    b = (rng.standard_normal((1, n, nrhs)) + 1j * rng.standard_normal((1, n, nrhs))).astype(np.complex64)
    db = CMatrices(b, n + 2)
    st = lib.aclsolverCpotrs(handle.value, 0, n, nrhs, da.tensor.data_ptr(), da.ld, db.tensor.data_ptr(), db.ld,
                             info.data_ptr())
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS and int(info.cpu()[0]) == 0
    assert cbits(db.read(), oracle.cpotrs_batched(want, b))


@pytest.mark.parametrize("upper", [False, True])
@pytest.mark.parametrize("n", [1, 7, 16, 17, 64, 100, 128, 140])
def test_cpotri_matches_the_solve_of_the_identity(handle, n, upper):
    """aclsolverCpotri: the selected triangle of A^-1 from a complex factor, in place, as the
    solve of L L^H X = I (the reference's cpotri, src/cpotri/arch35/cpotri.cpp) with this
    build's solve: bit for bit the oracle's cpotrs on the identity, Hermitian mirror in upper
    storage, padding untouched, close to the FP64 inverse."""
    import torch

    lib = aclsolver.library()
    a = hpd(1, n, seed=3 * n + int(upper))
    f, winfo = oracle.cpotrf_batched(a, upper=upper)
    assert winfo[0] == 0
    tri = np.triu(f[0]) if upper else np.tril(f[0])
    dm = CMatrices(tri[None], n + 1)
    lw = C.c_int(-1)
    assert lib.aclsolverCpotri_bufferSize(handle.value, int(upper), n, dm.table[0].item(), dm.ld,
                                         C.byref(lw)) == aclsolver.SUCCESS
    work = torch.empty(2 * max(1, lw.value), dtype=torch.float32, device="cuda")
    info = info_buffer(1)
    st = lib.aclsolverCpotri(handle.value, int(upper), n, dm.table[0].item(), dm.ld, work.data_ptr(), lw.value,
                             info.data_ptr())
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS and int(info.cpu()[0]) == 0
    got = dm.read()[0]
    x = oracle.cpotrs_batched(f, np.eye(n, dtype=np.complex64)[None], upper=upper)[0]
    want = np.triu(np.conj(x.T)) if upper else np.tril(x)
    got_tri = np.triu(got) if upper else np.tril(got)
    assert cbits(got_tri, want)
    inv64 = np.linalg.inv(a[0].astype(np.complex128))
    ref = np.triu(inv64) if upper else np.tril(inv64)
    assert np.abs(got_tri - ref).max() <= 1e-4 * np.abs(inv64).max()


def test_cpotri_invalid_diagonal(handle):
    import torch

    lib = aclsolver.library()
    n = 20
    f, _ = oracle.cpotrf_batched(hpd(1, n, seed=9))
    f = np.tril(f)
    f[0, 6, 6] = 1.0 + 0.5j  # a non-zero imaginary part on the diagonal
    dm = CMatrices(f, n)
    work = torch.empty(2 * n * n, dtype=torch.float32, device="cuda")
    info = info_buffer(1)
    st = lib.aclsolverCpotri(handle.value, 0, n, dm.table[0].item(), n, work.data_ptr(), n * n, info.data_ptr())
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS and int(info.cpu()[0]) == 7
    assert dm.unchanged()


@pytest.mark.parametrize("upper", [False, True])
@pytest.mark.parametrize("n", [241, 300, 521])
def test_cpotrf_large_over_the_whole_gpu(handle, n, upper):
    """Orders above the shared-memory block path: one matrix over the whole GPU (64-column
    panels, diagonal block / rows / trailing Hermitian update kernels), bit for bit the
    oracle's order, padding untouched, within 1e-5 of FP64 LAPACK."""
    lib = aclsolver.library()
    a = hpd(1, n, seed=n + int(upper))
    da = CMatrices(a, n + 3)
    info = info_buffer(1)
    st = lib.aclsolverCpotrf(handle.value, int(upper), n, da.tensor.data_ptr(), da.ld, None, 0, info.data_ptr())
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS and int(info.cpu()[0]) == 0
    got = da.read()
    want, winfo = oracle.cpotrf_batched(a, upper=upper)
    assert winfo[0] == 0
    assert cbits(got, want), "large complex factor differs from the oracle"
    tri = np.triu(got[0]) if upper else np.tril(got[0])
    gold = la.cholesky(a[0].astype(np.complex128), lower=not upper)
    assert np.abs(tri - gold).max() <= 1e-5 * max(1.0, np.abs(gold).max())


def test_cpotrf_large_batched_failures_keep_the_input_from_the_failed_column(handle):
    """CpotrfBatched above the block orders, one matrix at a time: a pivot failing in the
    first panel and one failing in a later panel (NaN) report their column; the completed
    columns hold the factor and the failed column onward the caller's input, as the
    oracle; a null slot gives -3."""
    lib = aclsolver.library()
    n = 260
    a = hpd(4, n, seed=21)
    a[1, 70, 70] = -1.0
    a[2, 255, 255] = np.nan
    dm = CMatrices(a, n)
    dm.table[3] = 0
    info = info_buffer(4)
    st = lib.aclsolverCpotrfBatched(handle.value, 0, n, dm.table.data_ptr(), n, info.data_ptr(), 4)
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS
    want, winfo = oracle.cpotrf_batched(a[:3])
    assert winfo.tolist() == [0, 71, 256]
    assert info.cpu().tolist() == [0, 71, 256, -3]
    assert cbits(dm.read()[:3], want)
