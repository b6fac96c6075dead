"""The oracle's complex LU restatement pinned without a GPU (the checker the GPU parity tests
trust):

  * the worked Cgetrs example of the reference API document (docs/zh/cgetrs.md);
  * the pivots of LAPACK's complex64 getrf on the reference's data recipes: both choose the
    largest |re| + |im| (PivotScore / icamax), earliest row on ties;
  * the reference's acceptance gates on its recipes: factor reconstruction
    (test/cgetrf/data/verify_result.py), solves against the reference's own numpy solver
    for trans 0, 1, 2 (test/utils/lu_verify_utils.py), inverses against numpy's
    (test/cgetri_batched/data/verify_result.py, test/cmatinv_batched/data/verify_result.py);
  * Divide against complex128 division across the exponent range, including the
    exponent-aligned branch, and exactly for the quotients that are representable;
  * the host-side argument ladders of the C entries that reject before any device work.

Fixtures: tests/golden/known_answers.json, tests/golden/complex_lu.npz (make_golden.py)."""

import ctypes as C
import json
from pathlib import Path

import numpy as np
import pytest

import oracle
from oracle import judges

GOLDEN = Path(__file__).resolve().parent / "golden"


def vectors():
    return np.load(GOLDEN / "complex_lu.npz")


def test_cgetrs_document_example():
    ka = json.loads((GOLDEN / "known_answers.json").read_text())["cgetrs_4x4"]
    lu = np.array(ka["lu"], dtype=np.float32).view(np.complex64).reshape(4, 4)  # row-major
    b = np.array(ka["b"], dtype=np.float32).view(np.complex64).reshape(4, 1)
    x = np.array(ka["x"], dtype=np.float32).view(np.complex64).reshape(4, 1)
    got = oracle.cgetrs_batched(lu[None], np.array([ka["ipiv"]], dtype=np.int32), b[None])[0]
    assert np.allclose(got, x, atol=1e-5)


@pytest.mark.parametrize("m,n", [(32, 32), (48, 64), (64, 48), (128, 128)])
def test_cgetrf_recipe_pivots_match_lapack_and_pass_the_gate(m, n):
    v = vectors()
    a = v[f"getrf_m{m}_n{n}_a"]
    lu, piv, info = oracle.cgetrf_batched(a[None])
    assert info[0] == 0
    assert np.array_equal(piv[0], v[f"getrf_m{m}_n{n}_lapack_ipiv"])
    assert judges.cgetrf_gate(a, lu[0], piv[0])


@pytest.mark.parametrize("n,nrhs", [(4, 1), (32, 32), (65, 3)])
@pytest.mark.parametrize("trans", [0, 1, 2])
def test_cgetrs_recipe_matches_the_reference_solver(n, nrhs, trans):
    v = vectors()
    key = f"getrs_n{n}_r{nrhs}"
    x = oracle.cgetrs_batched(v[key + "_lu"][None], v[key + "_ipiv"][None], v[key + "_b"][None], trans=trans)[0]
    assert judges.complex_solve_compare_ok(x, v[f"{key}_x{trans}"])


@pytest.mark.parametrize("n", [3, 32, 48])
def test_inverse_recipes_pass_the_reference_gate(n):
    v = vectors()
    a, golden = v[f"inverse_n{n}_a"], v[f"inverse_n{n}_golden"]
    direct, dinfo = oracle.cmatinv_batched(a)
    lu, piv, _ = oracle.cgetrf_batched(a)
    from_lu, linfo = oracle.cgetri_batched(lu, piv)
    assert np.all(dinfo == 0) and np.all(linfo == 0)
    for q in range(len(a)):
        assert judges.inverse_golden_ok(direct[q], golden[q])
        assert judges.inverse_golden_ok(from_lu[q], golden[q])
        assert judges.inverse_judge(a[q], from_lu[q])[0]


def test_divide_across_the_exponent_range():
    rng = np.random.default_rng(1)
    count = 20000
    ea = rng.uniform(-37, 37, size=(count, 2))
    eb = rng.uniform(-37, 37, size=(count, 2))
    a = (rng.standard_normal(count) * 10.0 ** ea[:, 0] + 1j * rng.standard_normal(count) * 10.0 ** ea[:, 1])
    b = (rng.standard_normal(count) * 10.0 ** eb[:, 0] + 1j * rng.standard_normal(count) * 10.0 ** eb[:, 1])
    a, b = a.astype(np.complex64), b.astype(np.complex64)
    q = oracle.cdivide(a, b).astype(np.complex128)
    exact = a.astype(np.complex128) / b.astype(np.complex128)
    normal = (np.abs(exact.real) > 1e-36) & (np.abs(exact.imag) > 1e-36) & (np.abs(exact) < 1e37)
    scale = np.abs(exact[normal])
    err = np.abs(q[normal] - exact[normal]) / scale
    assert err.max() < 3 * 2.0**-24 * 4  # a few ulps of the larger component


def test_divide_exact_quotients():
    # (a + bi) / (c + di) with small integer parts whose quotient is a dyadic rational
    a = np.array([6 + 8j, 1 + 0j, 0 + 2j, -3 - 4j, 5 + 0j], dtype=np.complex64)
    b = np.array([1 + 1j, 2 + 0j, 0 + 1j, 0 - 1j, 0 + 4j], dtype=np.complex64)
    q = oracle.cdivide(a, b)
    assert np.array_equal(q, (a.astype(np.complex128) / b.astype(np.complex128)).astype(np.complex64))


def test_lu_of_a_zero_matrix_reports_the_first_column():
    lu, piv, info = oracle.cgetrf_batched(np.zeros((1, 6, 6), dtype=np.complex64))
    assert info[0] == 1 and np.array_equal(piv[0], np.arange(1, 7))
    _, minfo = oracle.cmatinv_batched(np.zeros((1, 6, 6), dtype=np.complex64))
    assert minfo[0] == 1


def test_host_argument_ladders_without_a_gpu():
    import aclsolver

    lib = aclsolver.library()
    HANDLE_IS_NULLPTR, INVALID_PARAM = 9, 100000
    assert lib.aclsolverCgetrf(None, 4, 4, None, 4, None, None, None) == HANDLE_IS_NULLPTR
    assert lib.aclsolverCgetri(None, 4, None, 4, None, None, 16, None) == HANDLE_IS_NULLPTR
    assert lib.aclsolverCgetriBatched(None, 4, None, 4, None, None, 4, None, 1) == HANDLE_IS_NULLPTR
    assert lib.aclsolverCmatinvBatched(None, 4, None, 4, None, 4, None, 1) == HANDLE_IS_NULLPTR
    lw = C.c_int(-1)
    assert lib.aclsolverCgetri_bufferSize(None, 4, None, 4, C.byref(lw)) == HANDLE_IS_NULLPTR
    # Cgetrs checks its host arguments before touching any device
    a = np.zeros((4, 4), dtype=np.complex64)
    b = np.zeros((4, 1), dtype=np.complex64)
    piv = np.array([1, 2, 3, 4], dtype=np.int32)
    info = np.array([7], dtype=np.int32)
    call = lambda trans, n, nrhs, lda, ldb, p=piv: lib.aclsolverCgetrs(
        None, trans, n, nrhs, a.ctypes.data, lda, p.ctypes.data, b.ctypes.data, ldb, info.ctypes.data)
    assert call(3, 4, 1, 4, 1) == INVALID_PARAM
    assert call(0, 0, 1, 4, 1) == INVALID_PARAM
    assert call(0, 4, 1, 3, 1) == INVALID_PARAM
    assert call(0, 4, 2, 4, 1) == INVALID_PARAM
    assert call(0, 8193, 1, 8193, 1) == INVALID_PARAM
    assert info[0] == 7, "other argument errors leave info alone"
    bad = np.array([1, 5, 3, 4], dtype=np.int32)
    assert call(0, 4, 1, 4, 1, bad) == INVALID_PARAM and info[0] == -4
