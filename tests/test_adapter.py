"""The harness adapter protocol (include/solver_adapter.h; the reference's
test/sgetrf/solver_adapter.h, version 2): one library per real LU operation that an external
harness loads to drive the public entry point with compact row-major host buffers.

This file plays the harness.  Without a GPU: every adapter loads, exports the protocol's
functions, describes itself (operation, float32, device column-major, scalar or per-matrix
info, the address of the public function in libops_solver.so) and rejects malformed cases
before it touches the device.  On the GPU: create, reset, execute, synchronise, readback
and destroy for each operation, the outputs, info and pivots compared bit for bit with the
oracle, the padding sentinel and the 0xA5 fill of unwritten outputs checked, and a second
reset + execute giving the same bits (the reference's repeat check)."""

import ctypes as C
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
LIBDIR = ROOT / "ops-solver_b200" / "lib"
OPS = {"sgetrf": "aclsolverSgetrf", "sgetri": "aclsolverSgetri", "sgetri_batched": "aclsolverSgetriBatched",
       "smatinv_batched": "aclsolverSmatinvBatched"}
NAMES = {"sgetrf": b"sgetrf", "sgetri": b"sgetri", "sgetri_batched": b"sgetribatched",
         "smatinv_batched": b"smatinvbatched"}
OK, INVALID_CASE = 0, 1


class Desc(C.Structure):
    _fields_ = [("version", C.c_uint32), ("struct_size", C.c_uint32), ("op", C.c_char_p), ("dtype", C.c_char_p),
                ("dut_abi", C.c_char_p), ("dut_layout", C.c_char_p), ("info_kind", C.c_char_p),
                ("target_symbol", C.c_void_p)]


class Case(C.Structure):
    _fields_ = [("version", C.c_uint32), ("struct_size", C.c_uint32), ("n", C.c_int64), ("nrhs", C.c_int64),
                ("batch", C.c_int64), ("lda", C.c_int64), ("ldb", C.c_int64), ("uplo", C.c_char),
                ("info_probe", C.c_char_p), ("input_kind", C.c_char_p), ("a_bytes", C.c_size_t),
                ("b_bytes", C.c_size_t), ("out_bytes", C.c_size_t), ("info_count", C.c_size_t)]


class CaseV2(C.Structure):
    _fields_ = [("base", Case), ("m", C.c_int64), ("k", C.c_int64), ("ldc", C.c_int64), ("ldx", C.c_int64),
                ("side", C.c_char), ("trans", C.c_char), ("in_ipiv_count", C.c_size_t),
                ("in_tau_count", C.c_size_t), ("out_ipiv_count", C.c_size_t), ("out_tau_count", C.c_size_t)]


def adapter(op):
    lib = C.CDLL(str(LIBDIR / f"libsolver_adapter_{op}.so"))
    lib.solver_adapter_descriptor.restype = C.POINTER(Desc)
    lib.solver_adapter_create_v2.argtypes = [C.POINTER(CaseV2), C.c_void_p, C.c_void_p, C.POINTER(C.c_void_p)]
    lib.solver_adapter_reset_v2.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_void_p,
                                            C.c_size_t, C.c_void_p, C.c_size_t]
    lib.solver_adapter_execute.argtypes = [C.c_void_p, C.POINTER(C.c_int)]
    lib.solver_adapter_readback_v2.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t,
                                               C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t]
    lib.solver_adapter_destroy.argtypes = [C.c_void_p]
    return lib


def make_case(op, n, batch=1, m=None, lda=None, ldc=0, in_piv=0, out_piv=0):
    m = n if m is None else m
    c = CaseV2()
    c.base.version, c.base.struct_size = 2, C.sizeof(CaseV2)
    c.base.n, c.base.batch, c.base.lda = n, batch, lda if lda is not None else max(1, m)
    c.base.uplo = b"N"
    c.base.a_bytes = c.base.out_bytes = m * n * batch * 4
    c.base.info_count = batch if op in ("sgetri_batched", "smatinv_batched") else 1
    c.m, c.ldc = (m if op == "sgetrf" else 0), ldc
    c.in_ipiv_count, c.out_ipiv_count = in_piv, out_piv
    return c


@pytest.mark.parametrize("op", list(OPS))
def test_adapter_loads_and_describes_itself(op):
    import aclsolver

    lib = adapter(op)
    for fn in ("solver_adapter_descriptor", "solver_adapter_create_v2", "solver_adapter_reset_v2",
               "solver_adapter_execute", "solver_adapter_readback_v2", "solver_adapter_destroy"):
        assert hasattr(lib, fn), fn
    d = lib.solver_adapter_descriptor().contents
    assert d.version == 2 and d.struct_size == C.sizeof(Desc)
    assert d.op == NAMES[op] and d.dtype == b"float32" and d.dut_abi == b"device" and d.dut_layout == b"column_major"
    assert d.info_kind == (b"array" if "batched" in op else b"scalar")
    target = C.cast(getattr(aclsolver.library().lib, OPS[op]), C.c_void_p).value
    assert d.target_symbol == target, "the adapter must drive this library's public entry point"


@pytest.mark.parametrize("op", list(OPS))
def test_malformed_cases_are_rejected_before_any_device_work(op):
    lib = adapter(op)
    handle = C.c_void_p(0x1000)  # never dereferenced: validation fails first
    bad = []
    c = make_case(op, 8)
    c.base.version = 1
    bad.append(c)
    c = make_case(op, 8)
    c.base.a_bytes += 4
    bad.append(c)
    c = make_case(op, 8, lda=4)
    bad.append(c)
    c = make_case(op, 8)
    c.base.b_bytes = 16
    bad.append(c)
    if op == "smatinv_batched":
        bad.append(make_case(op, 33, ldc=33))
    if op in ("sgetri_batched", "smatinv_batched"):
        bad.append(make_case(op, 8, ldc=4))
    else:
        c = make_case(op, 8, batch=2)
        bad.append(c)
    for c in bad:
        state = C.c_void_p()
        assert lib.solver_adapter_create_v2(C.byref(c), handle, None, C.byref(state)) == INVALID_CASE
        assert lib.solver_adapter_destroy(state) == OK


def run_case(handle, op, a, case, ipiv_in=None, out_piv=0, repeat=False):
    """The harness sequence; returns (dut_status, out, info, ipiv_out)."""
    lib = adapter(op)
    state = C.c_void_p()
    st = lib.solver_adapter_create_v2(C.byref(case), handle.value, C.c_void_p(handle.stream.cuda_stream),
                                      C.byref(state))
    assert st == OK, st
    try:
        a = np.ascontiguousarray(a, dtype=np.float32)
        piv = None if ipiv_in is None else np.ascontiguousarray(ipiv_in, dtype=np.int32)
        out = np.full(a.shape, np.nan, dtype=np.float32)
        info = np.full(case.base.info_count, -12345, dtype=np.int32)
        ipiv = np.full(max(1, out_piv), -12345, dtype=np.int32)
        results = []
        for _ in range(2 if repeat else 1):
            assert lib.solver_adapter_reset_v2(state, a.ctypes.data, a.nbytes, None, 0,
                                               None if piv is None else piv.ctypes.data,
                                               0 if piv is None else piv.size, None, 0) == OK
            dut = C.c_int(-1)
            assert lib.solver_adapter_execute(state, C.byref(dut)) == OK
            handle.stream.synchronize()
            assert lib.solver_adapter_readback_v2(state, out.ctypes.data, out.nbytes, info.ctypes.data, info.size,
                                                  ipiv.ctypes.data if out_piv else None, out_piv, None, 0) == OK
            results.append((dut.value, out.copy(), info.copy(), ipiv[:out_piv].copy()))
        if repeat:
            assert results[0][0] == results[1][0]
            for x, y in zip(results[0][1:], results[1][1:]):
                assert np.array_equal(np.asarray(x).view(np.uint32), np.asarray(y).view(np.uint32)), "repeat differs"
        return results[-1]
    finally:
        assert lib.solver_adapter_destroy(state) == OK


def bits(x, y):
    return np.array_equal(np.asarray(x, dtype=np.float32).view(np.uint32), np.asarray(y, dtype=np.float32).view(np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("m,n,pad", [(64, 64, 0), (50, 30, 3), (300, 300, 5), (700, 600, 0)])
def test_sgetrf_adapter(handle, m, n, pad):
    import oracle

    rng = np.random.default_rng(m + n)
    a = rng.standard_normal((1, m, n)).astype(np.float32)
    steps = min(m, n)
    dut, out, info, ipiv = run_case(handle, "sgetrf", a, make_case("sgetrf", n, m=m, lda=m + pad, out_piv=steps),
                                    out_piv=steps, repeat=True)
    lu, wpiv, winfo = oracle.sgetrf_batched(a)
    assert dut == 0 and info.tolist() == winfo.tolist()
    assert np.array_equal(ipiv, wpiv.reshape(-1))
    assert bits(out, lu)


@pytest.mark.gpu
def test_sgetrf_adapter_null_pivots_and_singular_info(handle):
    import oracle

    n = 40
    a = np.random.default_rng(3).standard_normal((1, n, n)).astype(np.float32)
    a[0, :, 7] = 0.0
    dut, out, info, _ = run_case(handle, "sgetrf", a, make_case("sgetrf", n))
    lu, _, winfo = oracle.sgetrf_batched(a, pivoting=False)
    assert dut == 0 and info.tolist() == winfo.tolist() and info[0] == 8
    assert bits(out, lu)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [16, 64, 100])
def test_sgetri_adapter(handle, n):
    import oracle
    from oracle import judges

    rng = np.random.default_rng(n)
    a = rng.standard_normal((1, n, n)).astype(np.float32)
    lu, piv, _ = oracle.sgetrf_batched(a)
    dut, out, info, _ = run_case(handle, "sgetri", lu, make_case("sgetri", n, lda=n + 1, in_piv=n), ipiv_in=piv)
    assert dut == 0 and info.tolist() == [0]
    if n <= 64:
        inv, _ = oracle.sgetri_batched(lu, piv)
        assert bits(out, inv)
    else:
        assert judges.inverse_judge(a[0], out[0])[0]


@pytest.mark.gpu
def test_sgetri_batched_adapter(handle):
    import oracle

    n, batch = 64, 9
    rng = np.random.default_rng(1)
    a = rng.standard_normal((batch, n, n)).astype(np.float32)
    a[4, :, 11] = 0.0  # singular: info 12 and its output left alone
    lu, piv, _ = oracle.sgetrf_batched(a)
    dut, out, info, _ = run_case(handle, "sgetri_batched", lu,
                                 make_case("sgetri_batched", n, batch=batch, lda=n, ldc=n + 2, in_piv=n * batch),
                                 ipiv_in=piv, repeat=True)
    inv, winfo = oracle.sgetri_batched(lu, piv)
    assert dut == 0 and info.tolist() == winfo.tolist() and info[4] == 12
    ok = [q for q in range(batch) if q != 4]
    assert bits(out[ok], inv[ok])
    assert np.all(out[4].view(np.uint32) == 0xA5A5A5A5), "a failed matrix's output must stay unwritten"


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 5, 32])
def test_smatinv_batched_adapter(handle, n):
    import oracle

    batch = 40
    rng = np.random.default_rng(n)
    a = (rng.standard_normal((batch, n, n)) + 3 * np.eye(n)).astype(np.float32)
    dut, out, info, _ = run_case(handle, "smatinv_batched", a,
                                 make_case("smatinv_batched", n, batch=batch, lda=n + 1, ldc=n), repeat=True)
    lu, piv, _ = oracle.sgetrf_batched(a)
    inv, winfo = oracle.sgetri_batched(lu, piv)
    assert dut == 0 and info.tolist() == winfo.tolist()
    assert bits(out, inv)
