"""One batch of independent matrices split across GPUs, one process per GPU.

The batched entry points factor and solve independent matrices, so a batch shards with no
data-path exchange: rank r of W takes a contiguous slice of the batch, builds its own device
pointer tables over its slice and runs the ordinary entry points on its own stream.  The
only communication is the optional host gather of the per-matrix results (info, iteration
counts, backward errors) into batch order on rank 0, through torch.distributed (NCCL between
GPUs, gloo on CPU).  The reference runs on one device and has no counterpart; this module is
the host side of that split.
"""

import numpy as np


def shard_range(batch, rank, world):
    """The contiguous slice [start, start + count) of a batch of `batch` matrices that rank
    `rank` of `world` takes: sizes differ by at most one, the first `batch % world` ranks
    take the larger share."""
    if world < 1 or not 0 <= rank < world or batch < 0:
        raise ValueError(f"bad shard request: batch {batch}, rank {rank}, world {world}")
    base, extra = divmod(batch, world)
    start = rank * base + min(rank, extra)
    return start, base + (1 if rank < extra else 0)


def gather_to_root(local, batch, group=None, device=None):
    """Concatenates every rank's per-matrix values (a numpy array whose first axis runs over
    its slice, in slice order) into the batch order on rank 0; other ranks get None.  Every
    rank must call it (a collective).  `device`: where the exchange tensors live ("cuda" for
    NCCL, "cpu" for gloo; by default the backend's)."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    local = np.ascontiguousarray(local)
    start, count = shard_range(batch, rank, world)
    if local.shape[0] != count:
        raise ValueError(f"rank {rank} holds {local.shape[0]} values for a slice of {count}")
    if device is None:
        device = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    width = shard_range(batch, 0, world)[1]  # the largest slice
    buf = torch.zeros((max(1, width),) + local.shape[1:], dtype=torch.from_numpy(local[:0]).dtype, device=device)
    if count:
        buf[:count] = torch.from_numpy(local).to(device)
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    if rank != 0:
        return None
    out = [parts[r][: shard_range(batch, r, world)[1]].cpu().numpy() for r in range(world)]
    return np.concatenate(out) if out else local[:0]
