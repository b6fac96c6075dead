"""aclsolverSmatinvBatchedNoAlloc -- the small-matrix inverse for callers that cannot let the
library allocate device memory (hosts that own all device memory through their own pool,
allocation-free latency-critical loops): its pivots live in an array compiled into the
library instead of handle scratch.  Checked through the C ABI against aclsolverSmatinvBatched on the same
inputs, bit for bit (same kernels), on two calls in a row, plus its size limit.  The file
sorts last so that a run stopping at the first failure has run every other test first."""

import numpy as np
import pytest

import aclsolver
from helpers import DeviceMatrices, info_buffer, same_bits

pytestmark = pytest.mark.gpu


def run(handle, name, a, n):
    lib = aclsolver.library()
    count = len(a)
    da = DeviceMatrices(a, ld=n)
    dc = DeviceMatrices(np.zeros_like(a), ld=n + 1)
    info = info_buffer(count)
    st = getattr(lib, name)(handle.value, n, da.table_ptr, n, dc.table_ptr, n + 1, info.data_ptr(), count)
    handle.stream.synchronize()
    return st, dc.read(), info.cpu().numpy(), da.unchanged()


@pytest.mark.parametrize("n", [1, 5, 16, 32])
def test_no_alloc_matches_smatinv_on_two_calls(handle, n):
    rng = np.random.default_rng(7 * n)
    for call in range(2):
        a = (rng.standard_normal((300, n, n)) + 3 * np.eye(n)).astype(np.float32)
        a[5] = 0.0  # a singular slot: info > 0 and no output, identical in both entries
        st_ref, out_ref, info_ref, _ = run(handle, "aclsolverSmatinvBatched", a, n)
        st, out, info, kept = run(handle, "aclsolverSmatinvBatchedNoAlloc", a, n)
        assert st == st_ref == aclsolver.SUCCESS, call
        assert kept, "input matrices must be left unchanged"
        assert info.tolist() == info_ref.tolist()
        assert info[5] > 0 and np.count_nonzero(info) == 1
        assert same_bits(out, out_ref), call


def test_no_alloc_rejects_batches_beyond_the_fixed_array(handle):
    lib = aclsolver.library()
    n, count = 32, (1 << 20) // 32 + 1
    info = info_buffer(1)
    import torch

    table = torch.zeros(count, dtype=torch.int64, device="cuda")
    infos = info_buffer(count)
    st = lib.aclsolverSmatinvBatchedNoAlloc(handle.value, n, table.data_ptr(), n, table.data_ptr(), n,
                                           infos.data_ptr(), count)
    handle.stream.synchronize()
    assert st == aclsolver.INVALID_VALUE
    assert int(infos.cpu()[0]) == -7 and int(infos.cpu()[-1]) == -7
