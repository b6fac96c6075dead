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
from helpers import DeviceMatrices, device_ints, first_mismatch, info_buffer, same_bits

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
