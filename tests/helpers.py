"""Device-buffer helpers for the GPU parity tests.

Matrices travel the way the reference's runner lays them out (test/cholesky/runner.py:
87-165): column-major with a leading dimension larger than the order, the padding
filled with a sentinel that must survive the call, a device pointer table per batch and
info buffers pre-filled with a poison value.
"""

import numpy as np

SENTINEL = np.float32(-12345.125)
POISON = -777


class DeviceMatrices:
    """`count` column-major rows x cols float32 matrices in one device slab."""

    def __init__(self, mats, ld=None, device="cuda"):
        import torch

        from aclsolver import pointer_table

        mats = np.asarray(mats, dtype=np.float32)
        if mats.ndim == 2:
            mats = mats[None]
        self.count, self.rows, self.cols = mats.shape
        self.ld = max(1, self.rows) if ld is None else ld
        storage = np.full((self.count, max(self.cols, 1), self.ld), SENTINEL, dtype=np.float32)
        storage[:, : self.cols, : self.rows] = mats.transpose(0, 2, 1)
        self.initial = storage.copy()
        self.tensor = torch.from_numpy(storage.reshape(-1)).to(device)
        self.table = pointer_table(self.tensor, self.count, max(self.cols, 1) * self.ld * 4)

    @property
    def ptr(self):
        return self.tensor.data_ptr()

    @property
    def table_ptr(self):
        return self.table.data_ptr()

    def raw(self):
        return self.tensor.cpu().numpy().reshape(self.count, max(self.cols, 1), self.ld)

    def read(self, check_padding=True):
        raw = self.raw()
        if check_padding:
            assert np.all(raw[:, :, self.rows :] == SENTINEL), "leading-dimension padding overwritten"
        return np.ascontiguousarray(raw[:, : self.cols, : self.rows].transpose(0, 2, 1))

    def unchanged(self):
        return np.array_equal(self.raw().view(np.uint32), self.initial.view(np.uint32))


def device_ints(values, device="cuda"):
    import torch

    return torch.tensor(np.asarray(values, dtype=np.int32), device=device)


def info_buffer(count, device="cuda"):
    import torch

    return torch.full((max(1, count),), POISON, dtype=torch.int32, device=device)


def same_bits(a, b):
    """Bitwise equality of float32 arrays, any NaN matching any NaN."""
    a = np.asarray(a, dtype=np.float32)
    b = np.asarray(b, dtype=np.float32)
    if a.shape != b.shape:
        return False
    na, nb = np.isnan(a), np.isnan(b)
    if not np.array_equal(na, nb):
        return False
    return bool(np.array_equal(a.view(np.uint32)[~na], b.view(np.uint32)[~nb]))


def first_mismatch(a, b):
    a = np.asarray(a, dtype=np.float32)
    b = np.asarray(b, dtype=np.float32)
    diff = (a.view(np.uint32) != b.view(np.uint32)) & ~(np.isnan(a) & np.isnan(b))
    idx = np.argwhere(diff)
    if len(idx) == 0:
        return None
    i = tuple(idx[0])
    return i, float(a[i]), float(b[i]), int(diff.sum())


def spd_batch(count, n, seed, scale_by_n=True):
    """A = G G^T / n + I with G ~ N(0,1) (the Cholesky workload recipe)."""
    rng = np.random.default_rng(seed)
    g = rng.standard_normal((count, n, n), dtype=np.float32)
    a = np.matmul(g, g.transpose(0, 2, 1)) / (n if scale_by_n else 1) + np.eye(n, dtype=np.float32)
    return a.astype(np.float32)


def conditioned_batch(count, n, kappa, seed):
    """A = U diag(s) V^T with U, V Haar-random orthogonal (QR of N(0,1), signs fixed by R's
    diagonal) and s log-spaced from 1 to 1/kappa; FP32 matrices of 2-norm condition ~kappa."""
    rng = np.random.default_rng(seed)
    s = np.logspace(0.0, -np.log10(kappa), n)
    out = np.empty((count, n, n), dtype=np.float32)
    for q in range(count):
        u, ru = np.linalg.qr(rng.standard_normal((n, n)))
        v, rv = np.linalg.qr(rng.standard_normal((n, n)))
        u *= np.sign(np.diag(ru))
        v *= np.sign(np.diag(rv))
        out[q] = ((u * s) @ v.T).astype(np.float32)
    return out
