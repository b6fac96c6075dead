"""The C-ABI library: it loads without a GPU, exports every symbol the public headers
declare, and its host-only contracts hold (CPU only; no compute is launched)."""

import ctypes as C

import numpy as np
import pytest

import aclsolver


def test_library_loads_and_exports_every_declared_symbol():
    lib = aclsolver.library()
    declared = aclsolver.declared_symbols()
    assert len(declared) >= 19
    missing = [name for name in declared if getattr(lib.lib, name, None) is None]
    assert not missing, f"declared but not exported: {missing}"


def test_binding_covers_the_declared_entry_points():
    missing = set(aclsolver.declared_symbols()) - set(aclsolver.ARGTYPES)
    assert not missing, f"no ctypes signature for {sorted(missing)}"


def test_create_rejects_null_output_and_existing_handle():
    lib = aclsolver.library()
    assert lib.aclsolverCreate(None) == aclsolver.HANDLE_IS_NULLPTR
    existing = C.c_void_p(0x1234)
    assert lib.aclsolverCreate(C.byref(existing)) == aclsolver.INVALID_VALUE
    assert existing.value == 0x1234


@pytest.mark.parametrize(
    "name,args",
    [
        ("aclsolverDestroy", []),
        ("aclsolverSetStream", [None]),
        ("aclsolverSpotrfBatched", [0, 4, None, 4, None, 1]),
        ("aclsolverSpotrsBatched", [0, 4, 1, None, 4, None, 4, None, 1]),
        ("aclsolverSgetrf", [4, 4, None, 4, None, None, None]),
        ("aclsolverSgetriBatched", [4, None, 4, None, None, 4, None, 1]),
        ("aclsolverSmatinvBatched", [4, None, 4, None, 4, None, 1]),
        ("aclsolverSgetrfBatched", [4, None, 4, None, None, 1]),
    ],
)
def test_null_handle_is_reported(name, args):
    lib = aclsolver.library()
    assert getattr(lib, name)(None, *args) == aclsolver.HANDLE_IS_NULLPTR


@pytest.mark.parametrize(
    "name,args",
    [
        ("aclsolverSgetrsBatched", [0, 4, 1, None, 4, None, None, 4, None, 1]),
        ("aclsolverSgetrfBatchedMixed", [3, 4, None, 4, None, None, 1]),
        ("aclsolverSgesvIrBatched", [3, 4, 1, None, 4, None, 4, None, 4, 2, 1e-7, None, None, None, 1]),
        ("aclsolverSmatinvBatchedNoAlloc", [4, None, 4, None, 4, None, 1]),
        ("aclsolverSetDeviceChecks", [0]),
    ],
)
def test_null_handle_is_reported_by_the_additions(name, args):
    """The real-family additions follow the real family: HANDLE_IS_NULLPTR before any
    argument is looked at."""
    lib = aclsolver.library()
    assert getattr(lib, name)(None, *args) == aclsolver.HANDLE_IS_NULLPTR


@pytest.mark.parametrize(
    "name,args",
    [
        ("aclsolverCpotrfBatched", [0, 4, None, 4, None, 1]),
        ("aclsolverCpotrsBatched", [0, 4, 1, None, 4, None, 4, None, 1]),
        ("aclsolverCpotrsBatchedMultiRhs", [0, 4, 2, None, 4, None, 4, None, 1]),
    ],
)
def test_null_handle_in_the_complex_family(name, args):
    """The complex entries keep the reference's own convention for a null handle:
    NOT_INITIALIZED."""
    lib = aclsolver.library()
    assert getattr(lib, name)(None, *args) == aclsolver.NOT_INITIALIZED


def test_get_stream_contract():
    lib = aclsolver.library()
    out = C.c_void_p()
    assert lib.aclsolverGetStream(None, C.byref(out)) == aclsolver.HANDLE_IS_NULLPTR


def _sgetrs(trans, n, nrhs, lda, ldb, ipiv, a=True, b=True):
    lib = aclsolver.library()
    A = np.zeros(max(1, n * lda), dtype=np.float32)
    B = np.zeros(max(1, n * ldb), dtype=np.float32)
    P = np.asarray(ipiv, dtype=np.int32)
    info = np.array([123], dtype=np.int32)
    st = lib.aclsolverSgetrs(
        None, trans, n, nrhs, A.ctypes.data if a else None, lda, P.ctypes.data, B.ctypes.data if b else None, ldb,
        info.ctypes.data,
    )
    return st, int(info[0])


@pytest.mark.parametrize(
    "args",
    [
        (0, 0, 1, 1, 1),  # n = 0
        (0, 4, 0, 4, 1),  # nrhs = 0
        (0, 4, 1, 3, 1),  # lda < n
        (0, 4, 2, 4, 1),  # ldb < nrhs
        (0, 8193, 1, 8193, 1),  # n > 8192
        (2, 4, 1, 4, 1),  # trans not 0/1
        (0, 4, 1, 4 + 16384, 1),  # lda - n > 16383
    ],
)
def test_sgetrs_host_argument_checks(args):
    trans, n, nrhs, lda, ldb = args
    st, info = _sgetrs(trans, n, nrhs, lda, ldb, [1] * max(1, n))
    assert st == aclsolver.ACL_ERROR_INVALID_PARAM
    assert info == 123  # left unmodified for argument errors other than ipiv


def test_sgetrs_null_buffers():
    st, info = _sgetrs(0, 4, 1, 4, 1, [1, 2, 3, 4], a=False)
    assert st == aclsolver.ACL_ERROR_INVALID_PARAM


@pytest.mark.parametrize("ipiv", [[0, 2, 3, 4], [1, 2, 3, 5], [1, -1, 3, 4]])
def test_sgetrs_rejects_pivots_outside_range(ipiv):
    st, info = _sgetrs(0, 4, 1, 4, 1, ipiv)
    assert st == aclsolver.ACL_ERROR_INVALID_PARAM
    assert info == -4
