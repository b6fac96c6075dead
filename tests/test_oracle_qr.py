"""The oracle's real QR restatement pinned without a GPU:

  * R and tau against LAPACK sgeqrf (same sign convention: beta = -sign(alpha) ||x||);
  * the reference's Sgeqrf gate on the oracle's factor: ||R - Q^T A||_1 / (m ||A||_1 eps)
    <= max(5 ratio_cpu, 0.1), ratio_cpu from the reference's own CPU golden (QrCore::Geqr2,
    src/sgeqrf/kernel/householder.hpp, restated as orc_sgeqr2_golden) (test/sgeqrf/sgeqrf_test.cpp:16);
  * Sormqr (both sides, both operations) and Sorgqr against an explicit Q;
  * the reference's SSgels gates (test/sgels/sgels_test.cpp:16-24): SQRT16 for square
    systems, SQRT17 (normal-equation optimality) for overdetermined ones, each against the
    same chain on the CPU golden factor;
  * the host argument ladders of the QR entries that reject before any device work."""

import ctypes as C

import numpy as np
import pytest

import oracle
from oracle import judges

SHAPES = [(2, 2), (18, 8), (32, 4), (57, 57), (66, 8), (100, 33), (33, 100), (128, 128), (300, 70),
          (2000, 40)]  # the last: panels reduced in eight row segments


def rand(m, n, seed):
    return np.random.default_rng(seed).standard_normal((m, n)).astype(np.float32)


@pytest.mark.parametrize("m,n", SHAPES)
def test_sgeqrf_matches_lapack_convention_and_passes_the_gate(m, n):
    from scipy.linalg import lapack

    a = rand(m, n, m * 31 + n)
    qr, tau = oracle.sgeqrf(a)
    lq, ltau, _, info = lapack.sgeqrf(a)
    k = min(m, n)
    scale = np.abs(lq).max()
    assert np.abs(np.triu(qr[:k]) - np.triu(lq[:k])).max() <= 1e-5 * scale
    assert np.abs(tau - ltau[:k]).max() <= 1e-5
    golden, gtau = oracle.sgeqr2_golden(a)
    ratio = judges.qr_ratio(a, qr, tau)
    cpu = judges.qr_ratio(a, golden, gtau)
    assert ratio <= max(5 * cpu, 0.1), (ratio, cpu)


@pytest.mark.parametrize("m,n", [(40, 40), (90, 33), (33, 33), (70, 5)])
def test_sormqr_and_sorgqr_against_an_explicit_q(m, n):
    a = rand(m, n, m + n)
    qr, tau = oracle.sgeqrf(a)
    k = min(m, n)
    q = oracle.sorgqr(qr, tau, m)  # the full m x m Q
    assert np.abs(q.T.astype(np.float64) @ q - np.eye(m)).max() < 1e-5
    assert np.abs(q[:, :k].astype(np.float64) @ np.triu(qr[:k]) - a).max() < 1e-5 * np.abs(a).max() * m
    rng = np.random.default_rng(1)
    cl = rng.standard_normal((m, 6)).astype(np.float32)
    cr = rng.standard_normal((5, m)).astype(np.float32)
    assert np.abs(oracle.sormqr(0, 0, qr, tau, cl) - q @ cl).max() < 1e-4
    assert np.abs(oracle.sormqr(0, 1, qr, tau, cl) - q.T @ cl).max() < 1e-4
    assert np.abs(oracle.sormqr(1, 0, qr, tau, cr) - cr @ q).max() < 1e-4
    assert np.abs(oracle.sormqr(1, 1, qr, tau, cr) - cr @ q.T).max() < 1e-4


@pytest.mark.parametrize("m,n,nrhs", [(20, 20, 3), (64, 64, 1), (100, 40, 5), (300, 70, 8)])
def test_sgels_passes_the_reference_gates(m, n, nrhs):
    a = rand(m, n, m * 7 + n)
    b = rand(m, nrhs, nrhs)
    x, _, _ = oracle.sgels(a.copy(), b)
    # CPU chain on the reference's golden factor: Q^T B by reflectors, back substitution
    g, gtau = oracle.sgeqr2_golden(a)
    y = oracle.sormqr(0, 1, g, gtau, b)
    xc = np.linalg.solve(np.triu(g[:n, :n]).astype(np.float64), y[:n].astype(np.float64)).astype(np.float32)
    assert judges.gels_ok(a, b, x, xc)


def test_host_argument_ladders_without_a_gpu():
    import aclsolver

    lib = aclsolver.library()
    INVALID, NOT_SUPPORTED, NULL_HANDLE = 3, 7, 9
    lw = C.c_int(-1)
    assert lib.aclsolverSgeqrf_bufferSize(None, 10, 4, None, 10, C.byref(lw)) == 0 and lw.value == 2048
    assert lib.aclsolverSgeqrf_bufferSize(None, 0, 4, None, 1, C.byref(lw)) == 0 and lw.value == 0
    assert lib.aclsolverSgeqrf_bufferSize(None, 10, 4, None, 9, C.byref(lw)) == INVALID
    assert lib.aclsolverSgeqrf_bufferSize(None, 8193, 4, None, 8193, C.byref(lw)) == NOT_SUPPORTED
    assert lib.aclsolverSorgqr_bufferSize(None, 10, 6, 4, None, 10, None, C.byref(lw)) == 0 and lw.value == 1064
    assert lib.aclsolverSorgqr_bufferSize(None, 10, 11, 4, None, 10, None, C.byref(lw)) == INVALID
    assert lib.aclsolverSormqr_bufferSize(None, 0, 1, 10, 3, 4, None, 10, None, None, 10, C.byref(lw)) == 0
    assert lib.aclsolverSormqr_bufferSize(None, 2, 1, 10, 3, 4, None, 10, None, None, 10, C.byref(lw)) == INVALID
    assert lib.aclsolverSormqr_bufferSize(None, 1, 0, 5000, 4097, 4, None, 4097, None, None, 5000,
                                          C.byref(lw)) == NOT_SUPPORTED
    sz = C.c_size_t(1)
    assert lib.aclsolverSSgels_bufferSize(None, 10, 4, 1, None, 10, None, 10, None, 4, None, C.byref(sz)) == NULL_HANDLE
    info = C.c_int(0)
    assert lib.aclsolverSgeqrf(None, 4, 4, None, 4, None, None, 0, C.byref(info)) == NULL_HANDLE
    assert lib.aclsolverSgeqrf(None, 4, 4, None, 4, None, None, 0, None) == INVALID
    assert lib.aclsolverSSgels(None, 4, 4, 1, None, 4, None, 4, None, 4, None, 0, None, None) == INVALID


@pytest.mark.parametrize("direct", [0, 1])
def test_slarft_forms_the_block_reflector(direct):
    """I - V T V^T equals H(1)...H(k) (forward) or H(k)...H(1) (backward), the reference's
    Larft contract (householder.hpp:172-200 for the forward case)."""
    rng = np.random.default_rng(direct)
    n, k = 50, 9
    v = rng.standard_normal((n, k)).astype(np.float32)
    tau = rng.uniform(0.2, 1.8, k).astype(np.float32)
    tau[4] = 0.0
    full = np.zeros((n, k))
    for i in range(k):
        u = i if direct == 0 else n - k + i
        full[u, i] = 1.0
        if direct == 0:
            full[u + 1:, i] = v[u + 1:, i]
        else:
            full[:u, i] = v[:u, i]
    h = np.eye(n)
    for i in (range(k) if direct == 0 else reversed(range(k))):
        h = h @ (np.eye(n) - float(tau[i]) * np.outer(full[:, i], full[:, i]))
    t = oracle.slarft(direct, v, tau).astype(np.float64)
    assert np.abs(h - (np.eye(n) - full @ t @ full.T)).max() < 1e-4 * np.abs(h).max()
    assert np.all((np.tril(t, -1) if direct == 0 else np.triu(t, 1)) == 0)
