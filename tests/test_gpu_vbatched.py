"""Uneven-order batched complex Cholesky factor + solve (the persistent, size-bucketed,
graph-captured plan): bit-identical to the uniform-order entry points' arithmetic (the
oracle), per-matrix info, failures isolated, and repeatable replays."""

import ctypes as C

import numpy as np
import pytest

import aclsolver
import oracle
from oracle import judges
from helpers import info_buffer, same_bits

pytestmark = pytest.mark.gpu


def hpd(n, rng):
    g = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    return (g @ g.conj().T / max(n, 1) + np.eye(n)).astype(np.complex64)


class Uneven:
    """Matrices of different orders, each in its own padded device buffer."""

    def __init__(self, orders, nrhs, seed, pad=1):
        import torch

        rng = np.random.default_rng(seed)
        self.orders = list(orders)
        self.nrhs = nrhs
        self.a = [hpd(n, rng) for n in self.orders]
        self.b = [(rng.standard_normal((n, nrhs)) + 1j * rng.standard_normal((n, nrhs))).astype(np.complex64)
                  for n in self.orders]
        self.lda = [max(1, n + pad) for n in self.orders]
        self.ldb = [max(1, n + 2 * pad) for n in self.orders]
        self.da, self.db = [], []
        for q, n in enumerate(self.orders):
            sa = np.zeros((max(n, 1), self.lda[q]), dtype=np.complex64)
            sa[:n, :n] = self.a[q].T
            sb = np.zeros((max(nrhs, 1), self.ldb[q]), dtype=np.complex64)
            sb[:nrhs, :n] = self.b[q].T
            self.da.append(torch.from_numpy(sa.view(np.float32).reshape(-1).copy()).cuda())
            self.db.append(torch.from_numpy(sb.view(np.float32).reshape(-1).copy()).cuda())
        self.ta = torch.tensor([t.data_ptr() for t in self.da], dtype=torch.int64, device="cuda")
        self.tb = torch.tensor([t.data_ptr() for t in self.db], dtype=torch.int64, device="cuda")

    def factor(self, q):
        n = self.orders[q]
        raw = self.da[q].cpu().numpy().view(np.complex64).reshape(max(n, 1), self.lda[q])
        return np.ascontiguousarray(raw[:n, :n].T)

    def solution(self, q):
        n = self.orders[q]
        raw = self.db[q].cpu().numpy().view(np.complex64).reshape(max(self.nrhs, 1), self.ldb[q])
        return np.ascontiguousarray(raw[: self.nrhs, :n].T)


def plan(handle, u, autotune=1, uplo=0):
    lib = aclsolver.library()
    n = np.asarray(u.orders, dtype=np.int32)
    lda = np.asarray(u.lda, dtype=np.int32)
    ldb = np.asarray(u.ldb, dtype=np.int32)
    p = C.c_void_p()
    st = lib.aclsolverCposvVbatchedPlanCreate(handle.value, uplo, n.ctypes.data, lda.ctypes.data, ldb.ctypes.data,
                                             u.nrhs, len(u.orders), autotune, C.byref(p))
    assert st == aclsolver.SUCCESS
    return p


@pytest.mark.parametrize("seed", [0, 1])
def test_uneven_batch_matches_oracle(handle, seed, tmp_path, monkeypatch):
    monkeypatch.setenv("OPS_SOLVER_TUNE_CACHE", str(tmp_path / "tune.txt"))
    rng = np.random.default_rng(100 + seed)
    orders = rng.integers(1, 129, size=300).tolist() + [8, 16, 17, 32, 33, 128, 0]
    u = Uneven(orders, nrhs=4, seed=seed)
    p = plan(handle, u)
    lib = aclsolver.library()
    info = info_buffer(len(orders))
    st = lib.aclsolverCposvVbatched(handle.value, p, u.ta.data_ptr(), u.tb.data_ptr(), info.data_ptr())
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS
    assert np.all(info.cpu().numpy() == 0)
    for q, n in enumerate(orders):
        if n == 0:
            continue
        f, _ = oracle.cpotrf_batched(u.a[q][None])
        x = oracle.cpotrs_batched(f, u.b[q][None])
        got_f = u.factor(q)
        assert same_bits(np.ascontiguousarray(np.tril(got_f)).view(np.float32), np.ascontiguousarray(np.tril(f[0])).view(np.float32)), (q, n)
        assert same_bits(u.solution(q).view(np.float32), np.ascontiguousarray(x[0]).view(np.float32)), (q, n)
    ratios, cpu = [], []
    for q in range(0, len(orders), 7):
        if orders[q]:
            ratios.append(judges.complex_ratio("potrs", u.a[q], u.solution(q), False, u.b[q]))
            cpu.append(judges.complex_cpu_ratio("potrs", u.a[q], False, u.b[q]))
    assert not judges.residual_gate(ratios, cpu), judges.residual_gate(ratios, cpu)
    assert lib.aclsolverVbatchedPlanDestroy(p) == aclsolver.SUCCESS


def test_uneven_batch_failure_isolated_and_replay(handle, tmp_path, monkeypatch):
    monkeypatch.setenv("OPS_SOLVER_TUNE_CACHE", str(tmp_path / "tune.txt"))
    orders = [40, 5, 12, 90, 20, 3]
    u = Uneven(orders, nrhs=2, seed=3)
    u.a[3][10, 10] = -5.0  # order 90 fails at column 11 (when the trailing update keeps it negative)
    import torch

    sa = np.zeros((90, u.lda[3]), dtype=np.complex64)
    sa[:90, :90] = u.a[3].T
    u.da[3].copy_(torch.from_numpy(sa.view(np.float32).reshape(-1).copy()))
    p = plan(handle, u, autotune=0)
    lib = aclsolver.library()
    info = info_buffer(len(orders))
    b_before = u.solution(3).copy()
    st = lib.aclsolverCposvVbatched(handle.value, p, u.ta.data_ptr(), u.tb.data_ptr(), info.data_ptr())
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS
    _, winfo = oracle.cpotrf_batched(u.a[3][None])
    got = info.cpu().tolist()
    assert got[3] == int(winfo[0]) and got[3] > 0
    assert [v for i, v in enumerate(got) if i != 3] == [0] * 5
    assert np.array_equal(u.solution(3), b_before), "a failed matrix leaves its right-hand sides"
    # replay the captured graph on fresh inputs: identical bits
    first = [u.solution(q).copy() for q in range(len(orders))]
    for q, n in enumerate(orders):
        sb = np.zeros((2, u.ldb[q]), dtype=np.complex64)
        sb[:2, :n] = u.b[q].T
        u.db[q].copy_(torch.from_numpy(sb.view(np.float32).reshape(-1).copy()))
        sa = np.zeros((max(n, 1), u.lda[q]), dtype=np.complex64)
        sa[:n, :n] = u.a[q].T
        u.da[q].copy_(torch.from_numpy(sa.view(np.float32).reshape(-1).copy()))
    st = lib.aclsolverCposvVbatched(handle.value, p, u.ta.data_ptr(), u.tb.data_ptr(), info.data_ptr())
    handle.stream.synchronize()
    for q in range(len(orders)):
        assert np.array_equal(u.solution(q).view(np.uint32), first[q].view(np.uint32))
    lib.aclsolverVbatchedPlanDestroy(p)


def test_plan_argument_checks(handle):
    lib = aclsolver.library()
    p = C.c_void_p()
    n = np.asarray([4, 161], dtype=np.int32)
    ld = np.asarray([4, 161], dtype=np.int32)
    assert lib.aclsolverCposvVbatchedPlanCreate(handle.value, 0, n.ctypes.data, ld.ctypes.data, ld.ctypes.data, 1, 2,
                                               0, C.byref(p)) == aclsolver.INVALID_VALUE
    assert lib.aclsolverCposvVbatchedPlanCreate(None, 0, n.ctypes.data, ld.ctypes.data, ld.ctypes.data, 1, 2, 0,
                                               C.byref(p)) == aclsolver.NOT_INITIALIZED


def test_uneven_batch_full_workload(handle, tmp_path, monkeypatch):
    """The uneven-order workload at full size: 20,000 HPD matrices of orders U{8..128},
    A = G G^H / n + I (real and imaginary parts of G N(0,1)), 4 right-hand sides, one plan
    and one call.  Every factor and solution bit for bit against the oracle (grouped by
    order), info all 0, and the reference's residual gate on a sample."""
    import torch

    monkeypatch.setenv("OPS_SOLVER_TUNE_CACHE", str(tmp_path / "tune.txt"))
    count, nrhs = 20_000, 4
    rng = np.random.default_rng(2)
    orders = rng.integers(8, 129, size=count).astype(np.int32)
    a_off = np.zeros(count, dtype=np.int64)
    b_off = np.zeros(count, dtype=np.int64)
    a_off[1:] = np.cumsum(orders.astype(np.int64) ** 2)[:-1]
    b_off[1:] = np.cumsum(orders.astype(np.int64) * nrhs)[:-1]
    a_flat = np.empty(int((orders.astype(np.int64) ** 2).sum()), dtype=np.complex64)
    b_flat = ((rng.standard_normal(int(orders.sum()) * nrhs) + 1j * rng.standard_normal(int(orders.sum()) * nrhs))
              * np.sqrt(0.5)).astype(np.complex64)
    groups = {}
    for n in np.unique(orders):
        idx = np.nonzero(orders == n)[0]
        g = (rng.standard_normal((len(idx), n, n)) + 1j * rng.standard_normal((len(idx), n, n))).astype(np.complex64)
        m = (g @ np.conj(g.transpose(0, 2, 1)) / np.float32(n) + np.eye(n, dtype=np.complex64)).astype(np.complex64)
        groups[int(n)] = (idx, m)
        for k, q in enumerate(idx):
            a_flat[a_off[q]:a_off[q] + n * n] = m[k].T.reshape(-1)
    da = torch.from_numpy(a_flat.view(np.float32).copy()).cuda()
    db = torch.from_numpy(b_flat.view(np.float32).copy()).cuda()
    ta = torch.from_numpy(a_off * 8).cuda() + da.data_ptr()
    tb = torch.from_numpy(b_off * 8).cuda() + db.data_ptr()
    lib = aclsolver.library()
    ld = np.ascontiguousarray(orders)
    p = C.c_void_p()
    assert lib.aclsolverCposvVbatchedPlanCreate(handle.value, 0, ld.ctypes.data, ld.ctypes.data, ld.ctypes.data, nrhs,
                                               count, 1, C.byref(p)) == aclsolver.SUCCESS
    info = info_buffer(count)
    st = lib.aclsolverCposvVbatched(handle.value, p, ta.data_ptr(), tb.data_ptr(), info.data_ptr())
    handle.stream.synchronize()
    assert st == aclsolver.SUCCESS
    assert np.all(info.cpu().numpy() == 0)
    lib.aclsolverVbatchedPlanDestroy(p)
    fa = da.cpu().numpy().view(np.complex64)
    xb = db.cpu().numpy().view(np.complex64)
    ratios, cpu = [], []
    for n, (idx, m) in groups.items():
        bq = np.stack([b_flat[b_off[q]:b_off[q] + n * nrhs].reshape(nrhs, n).T for q in idx])
        f, winfo = oracle.cpotrf_batched(m)
        assert np.all(winfo == 0)
        x = oracle.cpotrs_batched(f, bq)
        got_f = np.ascontiguousarray(np.stack([fa[a_off[q]:a_off[q] + n * n].reshape(n, n).T for q in idx]))
        got_x = np.ascontiguousarray(np.stack([xb[b_off[q]:b_off[q] + n * nrhs].reshape(nrhs, n).T for q in idx]))
        assert same_bits(np.tril(got_f).view(np.float32), np.tril(f).view(np.float32)), n
        assert same_bits(got_x.view(np.float32), np.ascontiguousarray(x).view(np.float32)), n
        k = 0  # one matrix per order for the residual gate
        ratios.append(judges.complex_ratio("potrs", m[k], got_x[k], False, bq[k]))
        cpu.append(judges.complex_cpu_ratio("potrs", m[k], False, bq[k]))
    assert not judges.residual_gate(ratios, cpu), judges.residual_gate(ratios, cpu)
