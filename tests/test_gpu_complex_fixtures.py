"""The shapes the reference's complex Cholesky fixtures exercise (test/utils/cholesky/
fixtures.py:42-56 of the reference): its throughput batches (orders 73 and 95, 1,025
matrices), the diagonal-state orders 144 / 145 in batches of 33, the buffered orders 864,
865 and 1,023 in batches (here 3 of the reference's 17, to bound the oracle's CPU time), the
solve-transition orders 511..2049, the right-hand-side counts 0..128, the single-matrix
boundary 4095 / 4096 and the edge order 33.  Each result is bit for bit the oracle's where
the oracle finishes in seconds, and always inside the reference's residual gate
max(5 x CPU-LAPACK ratio, 3 x batch mean) computed in complex128."""

import numpy as np
import pytest

import aclsolver
import oracle
from oracle import judges
from helpers import info_buffer
from test_gpu_complex import CMatrices, cbits, hpd

pytestmark = pytest.mark.gpu


def hermitian(a, upper):
    return np.triu(a) + np.triu(a, 1).conj().T if upper else np.tril(a) + np.tril(a, -1).conj().T


def factor(handle, a, upper=False, pad=1):
    lib = aclsolver.library()
    count, n, _ = a.shape
    dm = CMatrices(a, n + pad)
    info = info_buffer(count)
    st = lib.aclsolverCpotrfBatched(handle.value, int(upper), n, dm.table.data_ptr(), dm.ld, info.data_ptr(), count)
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS
    return dm.read(), info.cpu().numpy()


def gate_factor(a, got, upper):
    ratios = [judges.complex_ratio("potrf", hermitian(a[q], upper), got[q], upper) for q in range(len(a))]
    cpu = [judges.complex_cpu_ratio("potrf", hermitian(a[q], upper), upper) for q in range(len(a))]
    return judges.residual_gate(ratios, cpu)


@pytest.mark.parametrize("n,batch,upper", [(73, 1025, False), (95, 1025, True), (144, 33, False), (145, 33, True),
                                           (33, 7, False), (864, 3, False), (865, 3, True), (1023, 3, False)])
def test_cpotrf_batched_fixture_shapes(handle, n, batch, upper):
    a = hpd(batch, n, seed=950 + n)
    got, info = factor(handle, a, upper)
    assert np.all(info == 0)
    want, winfo = oracle.cpotrf_batched(a, upper=upper)
    assert np.all(winfo == 0)
    assert cbits(got, want)
    check = range(batch) if batch <= 33 else range(0, batch, 64)  # the gate on a sample of the big batches
    sub = np.array([a[q] for q in check])
    assert not gate_factor(sub, np.array([got[q] for q in check]), upper)


@pytest.mark.parametrize("n", [511, 512, 513, 1024, 1025, 2049])
@pytest.mark.parametrize("nrhs", [1, 17])
def test_cpotrs_solve_transition_orders(handle, n, nrhs):
    """CpotrsBatched (nrhs 1) / CpotrsBatchedMultiRhs (17) of the oracle's factor, bit for bit
    its solve, inside the residual gate."""
    lib = aclsolver.library()
    a = hpd(1, n, seed=n + nrhs)
    f, winfo = oracle.cpotrf_batched(a)
    assert winfo[0] == 0
    rng = np.random.default_rng(n)
    b = (rng.standard_normal((1, n, nrhs)) + 1j * rng.standard_normal((1, n, nrhs))).astype(np.complex64)
    da, db = CMatrices(f, n), CMatrices(b, n + 2)
    info = info_buffer(1)
    fn = lib.aclsolverCpotrsBatched if nrhs == 1 else lib.aclsolverCpotrsBatchedMultiRhs
    st = fn(handle.value, 0, n, nrhs, da.table.data_ptr(), n, db.table.data_ptr(), db.ld, info.data_ptr(), 1)
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS and int(info.cpu()[0]) == 0
    x = db.read()
    assert cbits(x, oracle.cpotrs_batched(f, b))
    full = hermitian(a[0], False)
    ratio = judges.complex_ratio("potrs", full, x[0], False, b[0])
    cpu = judges.complex_cpu_ratio("potrs", full, False, b[0])
    assert not judges.residual_gate([ratio], [cpu])


@pytest.mark.parametrize("nrhs", [0, 8, 9, 16, 17, 128])
def test_cpotrs_single_rhs_counts(handle, nrhs):
    lib = aclsolver.library()
    n = 40
    a = hpd(1, n, seed=nrhs)
    f, _ = oracle.cpotrf_batched(a)
    rng = np.random.default_rng(nrhs)
    b = (rng.standard_normal((1, n, max(nrhs, 1))) + 1j * rng.standard_normal((1, n, max(nrhs, 1))))
    b = b[:, :, :nrhs].astype(np.complex64)
    da = CMatrices(f, n)
    db = CMatrices(b if nrhs else np.zeros((1, n, 1), np.complex64), n)
    info = info_buffer(1)
    st = lib.aclsolverCpotrs(handle.value, 0, n, nrhs, da.tensor.data_ptr(), n, db.tensor.data_ptr(), n,
                             info.data_ptr())
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS and int(info.cpu()[0]) == 0
    if nrhs:
        assert cbits(db.read(), oracle.cpotrs_batched(f, b))
    else:
        assert db.unchanged()


@pytest.mark.parametrize("n", [4095, 4096])
def test_cpotrf_single_boundary_orders(handle, n):
    """One matrix at the largest orders (the whole-GPU path): info 0, the diagonal real and
    positive, and the factor inside the residual gate against scipy's complex64 LAPACK (the
    oracle's CPU loop would take minutes at this order)."""
    lib = aclsolver.library()
    a = hpd(1, n, seed=n)
    da = CMatrices(a, n)
    info = info_buffer(1)
    st = lib.aclsolverCpotrf(handle.value, 0, n, da.tensor.data_ptr(), n, None, 0, info.data_ptr())
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS and int(info.cpu()[0]) == 0
    got = da.read()
    d = np.diagonal(got[0])
    assert np.all(d.real > 0) and np.all(d.imag == 0)
    assert not gate_factor(a, got, False)
