"""Real LU parity through the C ABI on the GPU: SgetrfBatched / Sgetrf (identical ipiv and
bit-identical factors), SgetrsBatched / Sgetrs, SgetriBatched / Sgetri, SmatinvBatched,
against the oracle, the reference's known answers and its validation contracts."""

import ctypes as C
import json
from pathlib import Path

import numpy as np
import pytest

import aclsolver
import oracle
from oracle import judges
from helpers import DeviceMatrices, device_ints, first_mismatch, info_buffer, same_bits

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
KA = json.loads((GOLDEN / "known_answers.json").read_text())
SIZES = [1, 2, 3, 5, 7, 8, 9, 15, 16, 17, 31, 32, 33, 40, 63, 64]


def gaussian(count, n, seed, m=None):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((count, m or n, n)).astype(np.float32)


def integer_matrices(count, n, seed):
    """Small integers (the reference's file-mode recipe, randint 1..10) force pivot ties."""
    rng = np.random.default_rng(seed)
    return rng.integers(1, 11, size=(count, n, n)).astype(np.float32)


def getrf_batched(handle, a, pivoting=True, pad=2):
    lib = aclsolver.library()
    count, n, _ = a.shape
    dm = DeviceMatrices(a, ld=n + pad)
    piv = device_ints(np.zeros(max(1, count * n))) if pivoting else None
    info = info_buffer(count)
    st = lib.aclsolverSgetrfBatched(handle.value, n, dm.table_ptr, dm.ld, None if piv is None else piv.data_ptr(),
                                   info.data_ptr(), count)
    handle.stream.synchronize()
    ipiv = piv.cpu().numpy()[: count * n].reshape(count, n) if pivoting else None
    return st, dm, ipiv, info.cpu().numpy()


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("kind", ["gaussian", "integer"])
def test_sgetrf_batched_matches_oracle(handle, n, kind):
    a = gaussian(9, n, seed=n) if kind == "gaussian" else integer_matrices(9, n, seed=n)
    st, dm, ipiv, info = getrf_batched(handle, a)
    assert st == aclsolver.SUCCESS
    lu, wpiv, winfo = oracle.sgetrf_batched(a)
    assert info.tolist() == winfo.tolist()
    assert np.array_equal(ipiv, wpiv), "pivot sequences differ"
    got = dm.read()
    assert same_bits(got, lu), first_mismatch(got, lu)


def test_sgetrf_batched_without_pivoting(handle):
    a = gaussian(5, 24, seed=4) + 8 * np.eye(24, dtype=np.float32)
    st, dm, _, info = getrf_batched(handle, a, pivoting=False)
    lu, _, winfo = oracle.sgetrf_batched(a, pivoting=False)
    assert st == aclsolver.SUCCESS and info.tolist() == winfo.tolist()
    assert same_bits(dm.read(), lu)


def test_sgetrf_batched_special_values(handle):
    n = 16
    a = gaussian(6, n, seed=9)
    a[0, :, 3] = 0.0  # zero column -> info 4, factorisation continues
    a[1, 5, 5] = np.nan
    a[2, 7, 2] = np.inf
    a[3] *= 1e-39  # subnormal entries
    a[4, :, 0] = 2.0  # all-equal first column: earliest row wins
    a[5, 0, 0] = -0.0
    st, dm, ipiv, info = getrf_batched(handle, a)
    lu, wpiv, winfo = oracle.sgetrf_batched(a)
    assert info.tolist() == winfo.tolist()
    assert info[0] == 4
    assert np.array_equal(ipiv, wpiv)
    assert same_bits(dm.read(), lu)


def test_sgetrf_batched_workload_size(handle):
    """4,096 matrices of 64 x 64, N(0,1) entries: exact ipiv and bit-identical factors."""
    a = gaussian(4096, 64, seed=1)
    st, dm, ipiv, info = getrf_batched(handle, a, pad=0)
    lu, wpiv, winfo = oracle.sgetrf_batched(a)
    assert st == aclsolver.SUCCESS and np.all(info == 0)
    assert np.array_equal(ipiv, wpiv)
    assert same_bits(dm.read(), lu)


@pytest.mark.parametrize("m,n", [(4, 4), (7, 5), (5, 7), (64, 64), (33, 20), (1, 9), (9, 1), (64, 3)])
def test_sgetrf_single(handle, m, n):
    lib = aclsolver.library()
    a = gaussian(1, n, seed=m * 100 + n, m=m)
    dm = DeviceMatrices(a, ld=m + 3)
    lw = C.c_int(-1)
    assert lib.aclsolverSgetrf_bufferSize(handle.value, m, n, dm.ptr, dm.ld, C.byref(lw)) == aclsolver.SUCCESS
    import torch

    work = torch.empty(max(1, lw.value), dtype=torch.float32, device="cuda")
    piv = device_ints(np.zeros(min(m, n)))
    info = info_buffer(1)
    st = lib.aclsolverSgetrf(handle.value, m, n, dm.ptr, dm.ld, work.data_ptr(), piv.data_ptr(), info.data_ptr())
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS
    lu, wpiv, winfo = oracle.sgetrf_batched(a)
    assert int(info.cpu()[0]) == winfo[0]
    assert piv.cpu().tolist() == wpiv[0].tolist()
    assert same_bits(dm.read(), lu)
    assert judges.lu_reconstruction_ok(a[0], dm.read()[0], wpiv[0])


@pytest.mark.parametrize("name", ["2x2 subnormal pivot", "2x2 normal-scale control", "513x1 subnormal pivot"])
def test_sgetrf_subnormal_pivot_cases(handle, name):
    """The reference's subnormal-pivot cases (test/sgetrf/sgetrf_subnormal_pivot_test.cpp:
    157-167): a 2 x 2 matrix of subnormal entries, its normal-scale control, and a 513 x 1
    column of subnormals (the tall, single-column case, here on the whole-GPU path); the
    factors equal the oracle's bit for bit and P A = L U holds to 1e-5 relative, as the
    reference's check asks."""
    import torch

    tiny = np.float32(1.0e-39)
    cases = {
        "2x2 subnormal pivot": (2, 2, [2 * tiny, tiny, tiny, 2 * tiny]),
        "2x2 normal-scale control": (2, 2, [4.0e-38, 2.0e-38, 2.0e-38, 4.0e-38]),
        "513x1 subnormal pivot": (513, 1, [tiny] * 513),
    }
    m, n, values = cases[name]
    a = np.asarray(values, dtype=np.float32).reshape(1, m, n)  # row-major values, as the reference lists them
    lib = aclsolver.library()
    dm = DeviceMatrices(a, ld=m)
    lw = C.c_int(-1)
    assert lib.aclsolverSgetrf_bufferSize(handle.value, m, n, dm.ptr, m, C.byref(lw)) == aclsolver.SUCCESS
    work = torch.empty(max(1, lw.value), dtype=torch.float32, device="cuda")
    piv = device_ints(np.zeros(min(m, n)))
    info = info_buffer(1)
    st = lib.aclsolverSgetrf(handle.value, m, n, dm.ptr, m, work.data_ptr(), piv.data_ptr(), info.data_ptr())
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS and int(info.cpu()[0]) == 0
    lu, wpiv, winfo = oracle.sgetrf_batched(a)
    assert winfo[0] == 0 and piv.cpu().tolist() == wpiv[0].tolist()
    got = dm.read()[0]
    assert same_bits(got, lu[0])
    # P A = L U in FP64, relative to max |A|
    k = min(m, n)
    low = np.tril(got.astype(np.float64), -1)[:, :k] + np.eye(m, k)
    up = np.triu(got.astype(np.float64))[:k, :]
    pa = a[0].astype(np.float64).copy()
    for i, p in enumerate(wpiv[0]):
        pa[[i, p - 1]] = pa[[p - 1, i]]
    resid = np.abs(pa - low @ up).max() / np.abs(a[0]).max()
    assert np.isfinite(resid) and resid <= 1e-5, resid


def test_sgetrf_known_answer(handle):
    lib = aclsolver.library()
    case = KA["sgetrf_4x4"]
    a = np.asarray(case["a"], dtype=np.float32).reshape(1, 4, 4)
    dm = DeviceMatrices(a, ld=4)
    import torch

    work = torch.empty(16, dtype=torch.float32, device="cuda")
    piv = device_ints([0, 0, 0, 0])
    info = info_buffer(1)
    st = lib.aclsolverSgetrf(handle.value, 4, 4, dm.ptr, 4, work.data_ptr(), piv.data_ptr(), info.data_ptr())
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS and int(info.cpu()[0]) == 0
    assert piv.cpu().tolist() == case["ipiv"]
    np.testing.assert_allclose(dm.read()[0], np.asarray(case["lu"]).reshape(4, 4), atol=5e-7)


@pytest.mark.parametrize("index", range(5))
def test_sgetrf_basic_cases(handle, index):
    """The reference's basic native cases: forced swaps, no pivoting, singular (INFO 2)."""
    case = json.loads((GOLDEN / "basic_lu_cases.json").read_text())[index]
    lib = aclsolver.library()
    import torch

    for q, mat in enumerate(case["a"]):
        a = np.asarray(mat, dtype=np.float32)[None]
        m, n = case["m"], case["n"]
        dm = DeviceMatrices(a, ld=m + 8)
        work = torch.empty(64, dtype=torch.float32, device="cuda")
        piv = device_ints(np.zeros(min(m, n))) if case["pivot"] else None
        info = info_buffer(1)
        st = lib.aclsolverSgetrf(handle.value, m, n, dm.ptr, dm.ld, work.data_ptr(),
                                 None if piv is None else piv.data_ptr(), info.data_ptr())
        handle.stream.synchronize()
        assert st == aclsolver.SUCCESS
        assert int(info.cpu()[0]) == case["info"][q]
        lu, wpiv, _ = oracle.sgetrf_batched(a, pivoting=case["pivot"])
        assert same_bits(dm.read(), lu)
        if piv is not None:
            assert piv.cpu().tolist() == wpiv[0].tolist()


def test_sgetrf_rejects_non_finite_input(handle):
    lib = aclsolver.library()
    import torch

    a = gaussian(1, 8, seed=2)
    a[0, 3, 4] = np.nan
    dm = DeviceMatrices(a, ld=8)
    work = torch.empty(64, dtype=torch.float32, device="cuda")
    info = info_buffer(1)
    st = lib.aclsolverSgetrf(handle.value, 8, 8, dm.ptr, 8, work.data_ptr(), None, info.data_ptr())
    handle.stream.synchronize()
    assert st == aclsolver.INVALID_VALUE
    assert int(info.cpu()[0]) == -3
    assert dm.unchanged()


def test_sgetrf_invalid_dimension_writes_info(handle):
    lib = aclsolver.library()
    info = info_buffer(1)
    st = lib.aclsolverSgetrf(handle.value, -1, 2, None, 1, None, None, info.data_ptr())
    handle.stream.synchronize()
    assert st == aclsolver.INVALID_VALUE and int(info.cpu()[0]) == -1


def getrs_batched(handle, lu, ipiv, b, trans=0, pad=1):
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


@pytest.mark.parametrize("trans", [0, 1])
@pytest.mark.parametrize("n,nrhs", [(1, 1), (4, 2), (8, 1), (17, 3), (32, 1), (33, 2), (64, 1), (64, 5)])
def test_sgetrs_batched_matches_oracle(handle, n, nrhs, trans):
    a = gaussian(6, n, seed=n + 7)
    lu, ipiv, _ = oracle.sgetrf_batched(a)
    b = gaussian(6, nrhs, seed=n + 8, m=n)
    st, da, db, info = getrs_batched(handle, lu, ipiv, b, trans)
    assert st == aclsolver.SUCCESS and np.all(info == 0)
    assert da.unchanged()
    want = oracle.sgetrs_batched(lu, ipiv, b, trans=trans)
    assert same_bits(db.read(), want), first_mismatch(db.read(), want)
    for q in range(6):
        assert judges.solve_compare_ok(db.read()[q], judges.solve_lu(lu[q], b[q], ipiv[q], trans))


def test_sgetrs_batched_bad_pivot(handle):
    a = gaussian(3, 8, seed=1)
    lu, ipiv, _ = oracle.sgetrf_batched(a)
    ipiv = ipiv.copy()
    ipiv[1, 4] = 2  # below k+1
    b = gaussian(3, 1, seed=2, m=8)
    st, da, db, info = getrs_batched(handle, lu, ipiv, b)
    assert info.tolist() == [0, -6, 0]
    assert np.array_equal(db.read()[1], b[1])


@pytest.mark.parametrize("key", ["n8_r1_t0", "n33_r3_t1", "n64_r4_t0", "n64_r1_t1"])
def test_sgetrs_host_buffers_against_reference_solver(handle, key):
    """The host-buffer, row-major aclsolverSgetrs against the reference's numpy solver."""
    g = np.load(GOLDEN / "solve_lu.npz")
    lu, ipiv, b, x = (g[key + s] for s in ("_lu", "_ipiv", "_b", "_x"))
    trans = int(key[-1])
    n, nrhs = b.shape
    lib = aclsolver.library()
    lda, ldb = n + 3, nrhs + 2
    A = np.zeros((n, lda), dtype=np.float32)
    A[:, :n] = lu  # row-major: A[r*lda + c] = LU(r, c)
    B = np.full((n, ldb), 7.5, dtype=np.float32)
    B[:, :nrhs] = b
    P = np.ascontiguousarray(ipiv, dtype=np.int32)
    info = np.array([99], dtype=np.int32)
    st = lib.aclsolverSgetrs(handle.value, trans, n, nrhs, A.ctypes.data, lda, P.ctypes.data, B.ctypes.data, ldb,
                             info.ctypes.data)
    assert st == 0 and info[0] == 0
    assert np.all(B[:, nrhs:] == 7.5)
    assert judges.solve_compare_ok(B[:, :nrhs], x)
    want = oracle.sgetrs_batched(lu[None], ipiv[None], b[None], trans=trans)[0]
    assert same_bits(B[:, :nrhs], want)


def test_sgetrs_known_answer(handle):
    case = KA["sgetrs_4x4"]
    lib = aclsolver.library()
    A = np.asarray(case["lu"], dtype=np.float32)
    B = np.asarray(case["b"], dtype=np.float32)
    P = np.asarray(case["ipiv"], dtype=np.int32)
    info = np.array([5], dtype=np.int32)
    st = lib.aclsolverSgetrs(handle.value, 0, 4, 1, A.ctypes.data, 4, P.ctypes.data, B.ctypes.data, 1,
                             info.ctypes.data)
    assert st == 0 and info[0] == 0
    np.testing.assert_allclose(B, case["x"], atol=1e-4)


def getri_batched(handle, lu, ipiv, pad=2):
    lib = aclsolver.library()
    count, n, _ = lu.shape
    da = DeviceMatrices(lu, ld=n + pad)
    dc = DeviceMatrices(np.zeros_like(lu), ld=n + pad + 1)
    piv = None if ipiv is None else device_ints(ipiv.reshape(-1))
    info = info_buffer(count)
    st = lib.aclsolverSgetriBatched(handle.value, n, da.table_ptr, da.ld, None if piv is None else piv.data_ptr(),
                                   dc.table_ptr, dc.ld, info.data_ptr(), count)
    handle.stream.synchronize()
    return st, da, dc, info.cpu().numpy()


@pytest.mark.parametrize("n", SIZES)
def test_sgetri_batched_matches_oracle(handle, n):
    a = gaussian(7, n, seed=3 * n)
    lu, ipiv, _ = oracle.sgetrf_batched(a)
    st, da, dc, info = getri_batched(handle, lu, ipiv)
    assert st == aclsolver.SUCCESS and np.all(info == 0)
    assert da.unchanged()
    want, winfo = oracle.sgetri_batched(lu, ipiv)
    assert same_bits(dc.read(), want), first_mismatch(dc.read(), want)


def test_sgetri_batched_workload_size(handle):
    a = gaussian(4096, 64, seed=1)
    lu, ipiv, _ = oracle.sgetrf_batched(a)
    st, da, dc, info = getri_batched(handle, lu, ipiv, pad=0)
    want, _ = oracle.sgetri_batched(lu, ipiv)
    assert st == aclsolver.SUCCESS and np.all(info == 0)
    assert same_bits(dc.read(), want)
    sample = np.arange(0, 4096, 41)
    eye = np.eye(64)
    for q in sample:
        assert np.abs(dc.read()[q].astype(np.float64) @ a[q].astype(np.float64) - eye).max() < 1e-2


def test_sgetri_batched_singular_slot_not_written(handle):
    a = gaussian(3, 12, seed=5)
    a[1, :, 6] = 0.0
    lu, ipiv, winfo = oracle.sgetrf_batched(a)
    st, da, dc, info = getri_batched(handle, lu, ipiv)
    assert info.tolist() == [0, int(winfo[1]), 0] and info[1] == 7
    assert np.all(dc.read()[1] == 0)


def test_sgetri_batched_contracts(handle):
    lib = aclsolver.library()
    a = gaussian(2, 6, seed=6)
    lu, ipiv, _ = oracle.sgetrf_batched(a)
    # non-finite factors are rejected synchronously with info = -2 in every slot
    bad = lu.copy()
    bad[1, 2, 2] = np.inf
    st, _, dc, info = getri_batched(handle, bad, ipiv)
    assert st == aclsolver.INVALID_VALUE and info.tolist() == [-2, -2]
    # a pivot outside [k+1, n] -> -4
    p = ipiv.copy()
    p[0, 3] = 1
    st, _, _, info = getri_batched(handle, lu, p)
    assert st == aclsolver.INVALID_VALUE and info.tolist() == [-4, -4]
    # overlapping outputs -> -5
    da = DeviceMatrices(lu, ld=6)
    dc = DeviceMatrices(np.zeros_like(lu), ld=6)
    dc.table[1] = dc.table[0]
    info_t = info_buffer(2)
    st = lib.aclsolverSgetriBatched(handle.value, 6, da.table_ptr, 6, None, dc.table_ptr, 6, info_t.data_ptr(), 2)
    handle.stream.synchronize()
    assert st == aclsolver.INVALID_VALUE and info_t.cpu().tolist() == [-5, -5]


def test_sgetri_single_in_place(handle):
    lib = aclsolver.library()
    import torch

    case = KA["sgetri_4x4"]
    a = np.asarray(case["a"], dtype=np.float32).reshape(1, 4, 4)
    lu, ipiv, _ = oracle.sgetrf_batched(a)
    dm = DeviceMatrices(lu, ld=5)
    lw = C.c_int(-1)
    assert lib.aclsolverSgetri_bufferSize(handle.value, 4, dm.ptr, 5, C.byref(lw)) == aclsolver.SUCCESS
    work = torch.empty(max(1, lw.value), dtype=torch.float32, device="cuda")
    piv = device_ints(ipiv[0])
    info = info_buffer(1)
    st = lib.aclsolverSgetri(handle.value, 4, dm.ptr, 5, piv.data_ptr(), work.data_ptr(), lw.value, info.data_ptr())
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS and int(info.cpu()[0]) == 0
    np.testing.assert_allclose(dm.read()[0], np.asarray(case["inverse"]).reshape(4, 4), atol=1e-6)
    want, _ = oracle.sgetri_batched(lu, ipiv)
    assert same_bits(dm.read(), want)


@pytest.mark.parametrize("n", [1, 2, 3, 8, 16, 17, 32])
def test_smatinv_batched(handle, n):
    lib = aclsolver.library()
    a = gaussian(9, n, seed=n + 40) + 3 * np.eye(n, dtype=np.float32)
    da = DeviceMatrices(a, ld=n)
    dc = DeviceMatrices(np.zeros_like(a), ld=n + 1)
    info = info_buffer(9)
    st = lib.aclsolverSmatinvBatched(handle.value, n, da.table_ptr, n, dc.table_ptr, n + 1, info.data_ptr(), 9)
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS and np.all(info.cpu().numpy() == 0)
    assert da.unchanged()
    lu, ipiv, _ = oracle.sgetrf_batched(a)
    want, _ = oracle.sgetri_batched(lu, ipiv)
    assert same_bits(dc.read(), want)


@pytest.mark.parametrize("n", [2, 5, 8, 16, 31, 32])
def test_smatinv_batched_passes_the_reference_inverse_judge(handle, n):
    """The reference's own acceptance for SmatinvBatched (verify_inverse: A @ X = I within
    rtol = atol = 5e-3, at most 1e-4 of the entries outside) on 512 N(0,1) matrices per
    order: its arithmetic on the target device is vector code with Newton steps that this
    build does not restate, so the contract with it is this judge; bit parity is held with
    the LU + vector-inverse order above."""
    lib = aclsolver.library()
    count = 512
    a = gaussian(count, n, seed=7 * n + 1)
    da = DeviceMatrices(a, ld=n)
    dc = DeviceMatrices(np.zeros_like(a), ld=n)
    info = info_buffer(count)
    st = lib.aclsolverSmatinvBatched(handle.value, n, da.table_ptr, n, dc.table_ptr, n, info.data_ptr(), count)
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS and np.all(info.cpu().numpy() == 0)
    x = dc.read()
    failed = [q for q in range(count) if not judges.inverse_judge(a[q], x[q])[0]]
    # the judge measures A X - I absolutely: an ill-conditioned draw can miss in exact FP32
    # arithmetic too, so the build must fail no matrix that FP32 LAPACK passes
    from scipy.linalg import lapack

    for q in failed:
        lu, piv, _ = lapack.sgetrf(a[q])
        inv, _ = lapack.sgetri(lu, piv)
        assert not judges.inverse_judge(a[q], inv)[0], (q, judges.inverse_judge(a[q], x[q]))


def test_smatinv_known_answer(handle):
    lib = aclsolver.library()
    case = KA["smatinv_2x2"]
    a = np.stack([np.asarray(m, dtype=np.float32).reshape(2, 2) for m in case["a"]])
    da = DeviceMatrices(a, ld=2)
    dc = DeviceMatrices(np.zeros_like(a), ld=2)
    info = info_buffer(2)
    st = lib.aclsolverSmatinvBatched(handle.value, 2, da.table_ptr, 2, dc.table_ptr, 2, info.data_ptr(), 2)
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS and info.cpu().tolist() == [0, 0]
    for q in range(2):
        np.testing.assert_array_equal(dc.read()[q], np.asarray(case["inverse"][q], dtype=np.float32).reshape(2, 2))


def test_smatinv_rejects_order_above_32(handle):
    lib = aclsolver.library()
    info = info_buffer(1)
    st = lib.aclsolverSmatinvBatched(handle.value, 33, None, 33, None, 33, info.data_ptr(), 1)
    handle.stream.synchronize()
    assert st == aclsolver.INVALID_VALUE and int(info.cpu()[0]) == -1
