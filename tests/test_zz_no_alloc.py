"""aclsolverSmatinvBatchedNoAlloc -- the small-matrix inverse for callers that cannot let the
library allocate device memory (hosts that own all device memory through their own pool,
allocation-free latency-critical loops): its pivots live in an array compiled into the
library instead of handle scratch.  Checked through the C ABI against aclsolverSmatinvBatched
on the same inputs, bit for bit (same kernels), on two calls in a row; that a call on a fresh
handle leaves the device's free memory unchanged; and its size and argument limits.  The
file sorts last so that a run stopping at the first failure has run every other test first."""

import numpy as np
import pytest

import aclsolver
from helpers import POISON, DeviceMatrices, info_buffer, same_bits

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


def test_no_alloc_on_a_fresh_handle_leaves_free_memory_unchanged(cuda):
    """The entry is called first on a new handle (no scratch leased yet); the device's free
    memory is the same before and after, so nothing was allocated on the caller's behalf.
    A first call on another handle loads the kernels and resolves the array beforehand."""
    import torch

    n, count = 32, 2000
    rng = np.random.default_rng(11)
    a = (rng.standard_normal((count, n, n)) + 3 * np.eye(n)).astype(np.float32)
    da = DeviceMatrices(a, ld=n)
    dc = DeviceMatrices(np.zeros_like(a), ld=n)
    info = info_buffer(count)
    lib = aclsolver.library()
    with aclsolver.Handle() as warm:
        assert lib.aclsolverSmatinvBatchedNoAlloc(warm.value, n, da.table_ptr, n, dc.table_ptr, n, info.data_ptr(),
                                                  count) == aclsolver.SUCCESS
        warm.stream.synchronize()
    expected = dc.read().copy()
    with aclsolver.Handle() as fresh:
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info()
        st = lib.aclsolverSmatinvBatchedNoAlloc(fresh.value, n, da.table_ptr, n, dc.table_ptr, n, info.data_ptr(),
                                                count)
        fresh.stream.synchronize()
        free1, _ = torch.cuda.mem_get_info()
    assert st == aclsolver.SUCCESS
    assert free1 == free0, f"free device memory changed by {free0 - free1} bytes"
    assert np.all(info.cpu().numpy() == 0)
    assert same_bits(dc.read(), expected)


def test_no_alloc_rejects_batches_beyond_the_fixed_array(handle):
    import torch

    lib = aclsolver.library()
    n, count = 32, (1 << 20) // 32 + 1
    table = torch.zeros(count, dtype=torch.int64, device="cuda")
    infos = info_buffer(count)
    st = lib.aclsolverSmatinvBatchedNoAlloc(handle.value, n, table.data_ptr(), n, table.data_ptr(), n,
                                           infos.data_ptr(), count)
    handle.stream.synchronize()
    assert st == aclsolver.INVALID_VALUE
    assert int(infos.cpu()[0]) == -7 and int(infos.cpu()[-1]) == -7


@pytest.mark.parametrize("n, count", [(32, 1 << 20), (1, 10_000_001)])
def test_no_alloc_short_info_buffer_is_not_written(handle, n, count):
    """An oversize batch (beyond the fixed array, or beyond the batched entries' 10^7 limit)
    with a one-entry info buffer: INVALID_VALUE, and info is left alone because it cannot
    hold batchSize entries."""
    import torch

    lib = aclsolver.library()
    table = torch.zeros(4, dtype=torch.int64, device="cuda")
    info = info_buffer(1)
    st = lib.aclsolverSmatinvBatchedNoAlloc(handle.value, n, table.data_ptr(), n, table.data_ptr(), n,
                                           info.data_ptr(), count)
    handle.stream.synchronize()
    assert st == aclsolver.INVALID_VALUE
    assert int(info.cpu()[0]) == POISON
