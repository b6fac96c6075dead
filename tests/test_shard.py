"""The multi-GPU split of one batch (aclsolver.shard): contiguous slices that cover the batch
exactly once, and the gather of per-matrix results into batch order on rank 0, run as two
gloo ranks on the CPU.  Each rank factors its slice with the oracle standing in for its GPU;
the gathered info and pivots must equal one unsharded factorisation of the whole batch."""

import os
import socket

import numpy as np
import pytest

from aclsolver.shard import gather_to_root, shard_range


@pytest.mark.parametrize("batch,world", [(0, 1), (1, 2), (7, 2), (256, 2), (10, 3), (4096, 8), (5, 8)])
def test_slices_cover_the_batch_once(batch, world):
    seen = []
    for r in range(world):
        start, count = shard_range(batch, r, world)
        assert count >= 0
        seen += list(range(start, start + count))
    assert seen == list(range(batch))
    counts = [shard_range(batch, r, world)[1] for r in range(world)]
    assert max(counts) - min(counts) <= 1


def test_bad_requests_raise():
    for args in ((4, 2, 2), (4, -1, 2), (4, 0, 0), (-1, 0, 1)):
        with pytest.raises(ValueError):
            shard_range(*args)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, batch, n, out):
    import torch.distributed as dist

    import oracle

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(5)
        a = rng.standard_normal((batch, n, n)).astype(np.float32)
        a[3, :, 2] = 0.0  # a singular matrix: info 3
        start, count = shard_range(batch, rank, world)
        _, ipiv, info = oracle.sgetrf_batched(a[start:start + count], threads=1)
        all_info = gather_to_root(info.astype(np.int32), batch)
        all_piv = gather_to_root(ipiv.astype(np.int32).reshape(count, n), batch)  # n pivots per matrix
        if rank == 0:
            np.savez(out, info=all_info, ipiv=all_piv)
        else:
            assert all_info is None and all_piv is None
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_gather_in_batch_order(tmp_path):
    import torch.multiprocessing as mp

    import oracle

    batch, n, world = 13, 12, 2
    out = str(tmp_path / "gathered.npz")
    mp.start_processes(_rank_main, args=(world, _free_port(), batch, n, out), nprocs=world, join=True,
                       start_method="spawn")
    got = np.load(out)
    rng = np.random.default_rng(5)
    a = rng.standard_normal((batch, n, n)).astype(np.float32)
    a[3, :, 2] = 0.0
    _, ipiv, info = oracle.sgetrf_batched(a, threads=1)
    assert got["info"].tolist() == info.tolist()
    assert got["info"][3] == 3
    assert np.array_equal(got["ipiv"], ipiv)
