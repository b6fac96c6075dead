"""The oracle pinned against the reference's golden vectors and judges (CPU only).

Pins: the worked examples of the reference API documents (known_answers.json), the
deterministic cases of the reference's native LU test with their INFO values
(basic_lu_cases.json), the reference's numpy LU solver outputs (solve_lu.npz) and the
reference residual judge's FP32-LAPACK ratios (cholesky_cpu_ratios.npz).  All fixtures
were produced by tests/golden/make_golden.py from the reference tree.
"""

import json
from pathlib import Path

import numpy as np
import pytest

import oracle
from oracle import judges

GOLDEN = Path(__file__).resolve().parent / "golden"
KA = json.loads((GOLDEN / "known_answers.json").read_text())


def rowmajor(v, n):
    return np.asarray(v, dtype=np.float32).reshape(n, n)


def test_sgetrf_known_answer():
    case = KA["sgetrf_4x4"]
    lu, ipiv, info = oracle.sgetrf_batched(rowmajor(case["a"], 4)[None])
    assert info[0] == 0
    assert ipiv[0].tolist() == case["ipiv"]
    np.testing.assert_allclose(lu[0], rowmajor(case["lu"], 4), rtol=0, atol=5e-7)


def test_sgetri_known_answer():
    case = KA["sgetri_4x4"]
    lu, ipiv, info = oracle.sgetrf_batched(rowmajor(case["a"], 4)[None])
    np.testing.assert_allclose(lu[0], rowmajor(case["lu"], 4), atol=5e-7)
    inv, info = oracle.sgetri_batched(lu, ipiv)
    assert info[0] == 0
    np.testing.assert_allclose(inv[0], rowmajor(case["inverse"], 4), atol=1e-6)


def test_sgetrs_known_answer():
    case = KA["sgetrs_4x4"]
    lu = rowmajor(case["lu"], 4)[None]
    b = np.asarray(case["b"], dtype=np.float32).reshape(1, 4, 1)
    x = oracle.sgetrs_batched(lu, np.asarray([case["ipiv"]], dtype=np.int32), b)
    np.testing.assert_allclose(x[0, :, 0], case["x"], atol=1e-4)


def test_spotrf_batched_known_answer():
    case = KA["spotrf_batched_4x4"]
    a = np.stack([rowmajor(m, 4) for m in case["a"]])
    f, info = oracle.spotrf_batched(a)
    assert info.tolist() == [0, 0]
    for q in range(2):
        np.testing.assert_allclose(np.tril(f[q]), rowmajor(case["l"][q], 4), atol=1e-7)
        # the unselected triangle is untouched
        np.testing.assert_array_equal(np.triu(f[q], 1), np.triu(a[q], 1))


def test_spotrs_known_answer():
    case = KA["spotrs_4x4"]
    a = rowmajor(case["a"], 4)[None]
    f, info = oracle.spotrf_batched(a)
    np.testing.assert_allclose(np.tril(f[0]), rowmajor(case["l"], 4), atol=1e-7)
    x = oracle.spotrs_batched(f, np.asarray(case["b"], dtype=np.float32).reshape(1, 4, 1), single=True)
    np.testing.assert_allclose(x[0, :, 0], case["x"], atol=2e-6)


def test_smatinv_known_answer():
    case = KA["smatinv_2x2"]
    a = np.stack([rowmajor(m, 2) for m in case["a"]])
    lu, ipiv, info = oracle.sgetrf_batched(a)
    inv, info = oracle.sgetri_batched(lu, ipiv)
    for q in range(2):
        np.testing.assert_array_equal(inv[q], rowmajor(case["inverse"][q], 2))


@pytest.mark.parametrize("index", range(5))
def test_basic_lu_cases(index):
    case = json.loads((GOLDEN / "basic_lu_cases.json").read_text())[index]
    a = np.asarray(case["a"], dtype=np.float32)
    lu, ipiv, info = oracle.sgetrf_batched(a, pivoting=case["pivot"])
    assert info.tolist() == case["info"]
    for q in range(len(a)):
        if case["info"][q]:
            continue
        assert judges.lu_reconstruction_ok(a[q], lu[q], ipiv[q] if case["pivot"] else None)
        if case["pivot"] and case["m"] > 1:
            assert ipiv[q][0] == 2  # the pre-swapped rows force a first interchange


SOLVE = np.load(GOLDEN / "solve_lu.npz")


@pytest.mark.parametrize("key", sorted({k.rsplit("_", 1)[0] for k in SOLVE.files}))
def test_sgetrs_against_reference_solver(key):
    lu, ipiv, b, x = (SOLVE[key + s] for s in ("_lu", "_ipiv", "_b", "_x"))
    trans = int(key[-1])
    got = oracle.sgetrs_batched(lu[None], ipiv[None], b[None], trans=trans)[0]
    assert judges.solve_compare_ok(got, x)
    # and the restated numpy solver agrees with the reference's
    assert judges.solve_compare_ok(judges.solve_lu(lu, b, ipiv, trans), x)


RATIOS = np.load(GOLDEN / "cholesky_cpu_ratios.npz")


@pytest.mark.parametrize("n", [1, 8, 9, 17, 32, 33, 64, 65])
def test_cholesky_passes_reference_gate(n):
    a, b, cpu = RATIOS[f"n{n}_a"], RATIOS[f"n{n}_b"], RATIOS[f"n{n}_ratio_cpu"]
    f, info = oracle.spotrf_batched(a)
    assert np.all(info == 0)
    x = oracle.spotrs_batched(f, b)
    for q in range(len(a)):
        rf = judges.cholesky_ratio("potrf", a[q], np.tril(f[q]))
        rs = judges.cholesky_ratio("potrs", a[q], x[q], b32=b[q])
        assert rf <= max(5 * cpu[q, 0], 3 * cpu[:, 0].mean())
        assert rs <= max(5 * cpu[q, 1], 3 * cpu[:, 1].mean())


@pytest.mark.parametrize("n", [3, 8, 12, 32, 40])
def test_cholesky_upper_mirrors_lower(n):
    rng = np.random.default_rng(n)
    g = rng.standard_normal((3, n, n)).astype(np.float32)
    a = (g @ g.transpose(0, 2, 1) / n + np.eye(n)).astype(np.float32)
    fl, _ = oracle.spotrf_batched(a, upper=False)
    fu, _ = oracle.spotrf_batched(a, upper=True)
    np.testing.assert_array_equal(np.tril(fl), np.transpose(np.triu(fu), (0, 2, 1)))


def test_cholesky_failure_keeps_unfinished_columns():
    n = 12
    a = np.eye(n, dtype=np.float32)[None].repeat(2, 0)
    a[0, 5, 5] = -1.0  # slot 0 fails at column 6
    a[1, 9, 9] = np.nan  # slot 1 fails at column 10 (NaN pivot)
    f, info = oracle.spotrf_batched(a)
    assert info.tolist() == [6, 10]
    np.testing.assert_array_equal(f[0][:, 5:], a[0][:, 5:])
    np.testing.assert_array_equal(f[1][:, 9:], a[1][:, 9:])


def test_lu_tie_rule_and_nan_rule():
    # equal magnitudes: the earliest row wins; -x ties with x
    a = np.array([[[1, 2], [-1, 3]]], dtype=np.float32).transpose(0, 2, 1)
    lu, ipiv, info = oracle.sgetrf_batched(np.array([[[1.0, 2.0], [-1.0, 3.0]]], dtype=np.float32))
    assert ipiv[0].tolist() == [1, 2]
    # a NaN on the diagonal keeps the row; a NaN elsewhere never wins
    lu, ipiv, info = oracle.sgetrf_batched(np.array([[[np.nan, 1.0], [5.0, 1.0]]], dtype=np.float32))
    assert ipiv[0][0] == 1
    lu, ipiv, info = oracle.sgetrf_batched(np.array([[[1.0, 1.0], [np.nan, 1.0], [3.0, 0.0]]], dtype=np.float32))
    assert ipiv[0][0] == 3


def test_lu_zero_pivot_continues():
    a = np.array([[[0.0, 1.0, 2.0], [0.0, 3.0, 4.0], [0.0, 5.0, 7.0]]], dtype=np.float32)
    lu, ipiv, info = oracle.sgetrf_batched(a)
    assert info[0] == 1  # first zero pivot, factorisation continues
    assert ipiv[0].tolist()[0] == 1


def test_residual_gate_flags_an_inflated_ratio():
    """The reference's batched gate max(5 x cpu, 3 x mean(cpu)): a device ratio planted above
    its threshold, and a non-finite one, are reported; the rest pass."""
    cpu = np.array([1.0, 2.0, 0.5, 0.5])
    ok = np.array([4.9, 9.9, 3.0, 0.1])
    assert judges.residual_gate(ok, cpu) == []
    bad = ok.copy()
    bad[2] = 3.1  # threshold max(2.5, 3 * 1.0) = 3.0
    bad[3] = np.inf
    assert [i for i, _, _ in judges.residual_gate(bad, cpu)] == [2, 3]


def test_inverse_judge_accepts_the_oracle_and_rejects_a_planted_error():
    rng = np.random.default_rng(3)
    a = (rng.standard_normal((1, 24, 24)) + 4 * np.eye(24)).astype(np.float32)
    lu, ipiv, _ = oracle.sgetrf_batched(a)
    x, _ = oracle.sgetri_batched(lu, ipiv)
    ok, ratio = judges.inverse_judge(a[0], x[0])
    assert ok and ratio == 0.0
    bad = x[0].copy()
    bad[3, 5] += 0.5  # a planted error spoils a row of A @ X
    ok, ratio = judges.inverse_judge(a[0], bad)
    assert not ok and ratio > 1e-4
