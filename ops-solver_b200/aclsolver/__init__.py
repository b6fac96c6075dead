"""ctypes binding of libops_solver.so, the B200 build of the aclsolver C ABI.

The binding mirrors how the reference's own test runner drives its library
(test/cholesky/runner.py:27-63): the C entry points are called through ctypes with
plain device addresses, and a tensor library supplies device buffers (torch on CUDA
here, torch_npu there).  It adds no compute of its own: every call goes to the CUDA
library, and loading fails loudly when the library has not been built.
"""

import ctypes as C
import os
from pathlib import Path

HERE = Path(__file__).resolve().parent
PACKAGE = HERE.parent
LIBRARY = PACKAGE / "lib" / "libops_solver.so"
INCLUDE = PACKAGE.parent / "include"

VP = C.c_void_p
I32 = C.c_int
I64 = C.c_int64
U64 = C.c_uint64

# Status codes (include/cann_ops_solver_common.h).
SUCCESS = 0
NOT_INITIALIZED = 1
ALLOC_FAILED = 2
INVALID_VALUE = 3
EXECUTION_FAILED = 5
INTERNAL_ERROR = 6
NOT_SUPPORTED = 7
HANDLE_IS_NULLPTR = 9
ACL_ERROR_INVALID_PARAM = 100000

LOWER = 0
UPPER = 1
OP_N = 0
OP_T = 1
FACTOR_FP32 = 0
FACTOR_BF16 = 1
FACTOR_BF16X3 = 3

_QUERY = [VP, I32, I32, VP, I32, C.POINTER(I32)]
ARGTYPES = {
    "aclsolverCreate": [C.POINTER(VP)],
    "aclsolverDestroy": [VP],
    "aclsolverSetStream": [VP, VP],
    "aclsolverGetStream": [VP, C.POINTER(VP)],
    # real Cholesky
    "aclsolverSpotrf_bufferSize": _QUERY,
    "aclsolverSpotri_bufferSize": _QUERY,
    "aclsolverSpotrf": [VP, I32, I32, VP, I32, VP, I32, VP],
    "aclsolverSpotri": [VP, I32, I32, VP, I32, VP, I32, VP],
    "aclsolverSpotrs": [VP, I32, I32, I32, VP, I32, VP, I32, VP],
    "aclsolverSpotrfBatched": [VP, I32, I32, VP, I32, VP, I32],
    "aclsolverSpotrsBatched": [VP, I32, I32, I32, VP, I32, VP, I32, VP, I32],
    # complex Cholesky
    "aclsolverCpotrf_bufferSize": _QUERY,
    "aclsolverCpotrf": [VP, I32, I32, VP, I32, VP, I32, VP],
    "aclsolverCpotrs": [VP, I32, I32, I32, VP, I32, VP, I32, VP],
    "aclsolverCpotri_bufferSize": _QUERY,
    "aclsolverCpotri": [VP, I32, I32, VP, I32, VP, I32, VP],
    "aclsolverCpotrfBatched": [VP, I32, I32, VP, I32, VP, I32],
    "aclsolverCpotrsBatched": [VP, I32, I32, I32, VP, I32, VP, I32, VP, I32],
    # real LU
    "aclsolverSgetrf_bufferSize": [VP, I32, I32, VP, I32, C.POINTER(I32)],
    "aclsolverSgetrf": [VP, I32, I32, VP, I32, VP, VP, VP],
    "aclsolverSgetri_bufferSize": [VP, I32, VP, I32, C.POINTER(I32)],
    "aclsolverSgetri": [VP, I32, VP, I32, VP, VP, I32, VP],
    "aclsolverSgetriBatched": [VP, I32, VP, I32, VP, VP, I32, VP, I32],
    "aclsolverSmatinvBatched": [VP, I32, VP, I32, VP, I32, VP, I32],
    "aclsolverSgetrs": [VP, U64, I64, I64, VP, I64, VP, VP, I64, VP],
    "aclsolverCgetrf_bufferSize": [VP, I32, I32, VP, I32, C.POINTER(I32)],
    "aclsolverCgetrf": [VP, I32, I32, VP, I32, VP, VP, VP],
    "aclsolverCgetri_bufferSize": [VP, I32, VP, I32, C.POINTER(I32)],
    "aclsolverCgetri": [VP, I32, VP, I32, VP, VP, I32, VP],
    "aclsolverCgetriBatched": [VP, I32, VP, I32, VP, VP, I32, VP, I32],
    "aclsolverCmatinvBatched": [VP, I32, VP, I32, VP, I32, VP, I32],
    "aclsolverCgetrs": [VP, U64, I64, I64, VP, I64, VP, VP, I64, VP],
    "aclsolverSgeqrf_bufferSize": [VP, I32, I32, VP, I32, C.POINTER(I32)],
    "aclsolverSgeqrf": [VP, I32, I32, VP, I32, VP, VP, I32, VP],
    "aclsolverSorgqr_bufferSize": [VP, I32, I32, I32, VP, I32, VP, C.POINTER(I32)],
    "aclsolverSorgqr": [VP, I32, I32, I32, VP, I32, VP, VP, I32, VP],
    "aclsolverSormqr_bufferSize": [VP, I32, I32, I32, I32, I32, VP, I32, VP, VP, I32, C.POINTER(I32)],
    "aclsolverSormqr": [VP, I32, I32, I32, I32, I32, VP, I32, VP, VP, I32, VP, I32, VP],
    "aclsolverXlarft_bufferSize": [VP, VP, I32, I32, I64, I64, I32, VP, I64, I32, VP, I32, VP, I64, I32,
                                   C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)],
    "aclsolverXlarft": [VP, VP, I32, I32, I64, I64, I32, VP, I64, I32, VP, I32, VP, I64, I32, VP, C.c_size_t, VP,
                        C.c_size_t],
    "aclsolverSSgels_bufferSize": [VP, I32, I32, I32, VP, I32, VP, I32, VP, I32, VP, C.POINTER(C.c_size_t)],
    "aclsolverSSgels": [VP, I32, I32, I32, VP, I32, VP, I32, VP, I32, VP, C.c_size_t, C.POINTER(I32), VP],
    "aclsolverCgeqrf_bufferSize": [VP, I32, I32, VP, I32, C.POINTER(I32)],
    "aclsolverCgeqrf": [VP, I32, I32, VP, I32, VP, VP, I32, VP],
    "aclsolverCungqr_bufferSize": [VP, I32, I32, I32, VP, I32, VP, C.POINTER(I32)],
    "aclsolverCungqr": [VP, I32, I32, I32, VP, I32, VP, VP, I32, VP],
    "aclsolverCunmqr_bufferSize": [VP, I32, I32, I32, I32, I32, VP, I32, VP, VP, I32, C.POINTER(I32)],
    "aclsolverCunmqr": [VP, I32, I32, I32, I32, I32, VP, I32, VP, VP, I32, VP, I32, VP],
    "aclsolverCCgels_bufferSize": [VP, I32, I32, I32, VP, I32, VP, I32, VP, I32, VP, C.POINTER(C.c_size_t)],
    "aclsolverCCgels": [VP, I32, I32, I32, VP, I32, VP, I32, VP, I32, VP, C.c_size_t, C.POINTER(I32), VP],
    # additions of this build
    "aclsolverSetDeviceChecks": [VP, I32],
    "aclsolverGetDeviceChecks": [VP, C.POINTER(I32)],
    "aclsolverSgetrfBatched": [VP, I32, VP, I32, VP, VP, I32],
    "aclsolverSgetrsBatched": [VP, I32, I32, I32, VP, I32, VP, VP, I32, VP, I32],
    "aclsolverCpotrsBatchedMultiRhs": [VP, I32, I32, I32, VP, I32, VP, I32, VP, I32],
    "aclsolverCposvVbatchedPlanCreate": [VP, I32, VP, VP, VP, I32, I32, I32, C.POINTER(VP)],
    "aclsolverCposvVbatched": [VP, VP, VP, VP, VP],
    "aclsolverVbatchedPlanDestroy": [VP],
    "aclsolverSmatinvBatchedNoAlloc": [VP, I32, VP, I32, VP, I32, VP, I32],
    "aclsolverSgetrfBatchedMixed": [VP, I32, I32, VP, I32, VP, VP, I32],
    "aclsolverSgesvIrBatched": [VP, I32, I32, I32, VP, I32, VP, I32, VP, I32, I32, C.c_double, VP, VP, VP, I32],
}


def declared_symbols():
    """Names of every function the public headers in include/ declare."""
    import re

    names = []
    for header in sorted(INCLUDE.glob("*.h")):
        text = header.read_text()
        names += re.findall(r"\b(?:aclsolverStatus_t|aclError)\s+(aclsolver\w+)\s*\(", text)
    return sorted(set(names))


class Library:
    """The loaded shared library with argument types declared for every entry point."""

    def __init__(self, path=None):
        path = Path(path or os.environ.get("OPS_SOLVER_LIBRARY", LIBRARY))
        if not path.exists():
            raise RuntimeError(
                f"{path} is missing: build it with `make -C ops-solver_b200` "
                "(or __graft_entry__.build())"
            )
        self.path = path
        self.lib = C.CDLL(str(path))
        for name, args in ARGTYPES.items():
            fn = getattr(self.lib, name, None)
            if fn is None:
                continue
            fn.argtypes = args
            fn.restype = I32

    def __getattr__(self, name):
        return getattr(self.lib, name)


_LIBRARY = None


def library():
    global _LIBRARY
    if _LIBRARY is None:
        _LIBRARY = Library()
    return _LIBRARY


class Handle:
    """An aclsolver handle bound to a CUDA stream (torch's current stream by default)."""

    def __init__(self, stream=None):
        import torch

        self.lib = library()
        self.value = VP()
        status = self.lib.aclsolverCreate(C.byref(self.value))
        if status != SUCCESS:
            raise RuntimeError(f"aclsolverCreate failed with status {status}")
        self.stream = stream if stream is not None else torch.cuda.current_stream()
        check(self.lib.aclsolverSetStream(self.value, self.stream.cuda_stream))

    def close(self):
        if self.value:
            self.stream.synchronize()
            check(self.lib.aclsolverDestroy(self.value))
            self.value = VP()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def check(status):
    if status != SUCCESS:
        raise RuntimeError(f"aclsolver status {status}")
    return status


def pointer_table(base, count, stride_bytes):
    """Device int64 table of `count` addresses base + q * stride_bytes (q = 0..count-1)."""
    import torch

    idx = torch.arange(count, dtype=torch.int64, device=base.device)
    return idx * int(stride_bytes) + int(base.data_ptr())


def ptr(t):
    """Device address of a tensor (None -> NULL)."""
    return None if t is None else t.data_ptr()
