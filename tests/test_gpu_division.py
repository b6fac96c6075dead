"""The division by a known reciprocal (Markstein's correction, `div_by` in common.cuh) that
the exact solves and panels use in place of the IEEE division: bit for bit IEEE float32
round-to-nearest division (numpy's) on random operands over the whole exponent range, on
operands built to land next to rounding boundaries, and on the special values that take the
IEEE path."""

import ctypes as C

import numpy as np
import pytest
import torch

import aclsolver

pytestmark = pytest.mark.gpu


SELFTEST = aclsolver.LIBRARY.parent / "libops_solver_selftest.so"


def gpu_divide(x, d):
    # the helper is exported by a test-only library built beside the product one
    assert SELFTEST.exists(), f"{SELFTEST} is missing: build it with `make -C ops-solver_b200`"
    fn = C.CDLL(str(SELFTEST)).ops_solver_selftest_divide
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_longlong]
    fn.restype = C.c_int
    xd = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float32)).cuda()
    dd = torch.from_numpy(np.ascontiguousarray(d, dtype=np.float32)).cuda()
    qd = torch.empty_like(xd)
    assert fn(xd.data_ptr(), dd.data_ptr(), qd.data_ptr(), xd.numel()) == 0
    return qd.cpu().numpy()


def check(x, d):
    with np.errstate(all="ignore"):
        want = (x / d).astype(np.float32)
    got = gpu_divide(x, d)
    same = (got.view(np.uint32) == want.view(np.uint32)) | (np.isnan(got) & np.isnan(want))
    bad = np.flatnonzero(~same)
    assert bad.size == 0, [(float(x[i]), float(d[i]), float(got[i]), float(want[i])) for i in bad[:5]]


def random_floats(rng, count, emin, emax):
    sig = rng.integers(1 << 23, 1 << 24, count, dtype=np.int64).astype(np.float64)
    e = rng.integers(emin, emax + 1, count)
    s = np.where(rng.random(count) < 0.5, -1.0, 1.0)
    return (s * np.ldexp(sig, e - 23)).astype(np.float32)


def test_random_operands(cuda):
    rng = np.random.default_rng(1)
    n = 1 << 24
    check(random_floats(rng, n, -70, 70), random_floats(rng, n, -70, 70))


def test_near_rounding_boundaries(cuda):
    """x = d (q + h ulp(q)) rounded, for h near 1/2: quotients next to a midpoint."""
    rng = np.random.default_rng(2)
    n = 1 << 22
    d = random_floats(rng, n, -20, 20)
    q = random_floats(rng, n, -20, 20)
    ulp = np.spacing(np.abs(q)).astype(np.float64)
    h = 0.5 + rng.integers(-4, 5, n) * 2.0 ** -26
    x = (d.astype(np.float64) * (q.astype(np.float64) + np.sign(q) * h * ulp)).astype(np.float32)
    check(x, d)
    # all-ones and power-of-two significands
    ones = np.float32(np.nextafter(np.float32(2.0), np.float32(0.0)))
    k = rng.integers(-30, 30, n)
    d2 = np.where(rng.random(n) < 0.5, np.ldexp(ones, k), np.ldexp(np.float32(1.0), k)).astype(np.float32)
    check(x, d2)
    check(d2, d)


def test_special_operands(cuda):
    specials = np.array([0.0, -0.0, 1.0, -1.0, np.inf, -np.inf, np.nan, 1e-45, -1e-45, 1e-40, 1.1754944e-38,
                         3.4028235e38, -3.4028235e38, 2.0 ** -60, 2.0 ** 60, 2.0 ** -61, 2.0 ** 61, 0.75, 3.0],
                        dtype=np.float32)
    x, d = np.meshgrid(specials, specials)
    check(x.ravel(), d.ravel())
    rng = np.random.default_rng(3)
    n = 1 << 20
    check(random_floats(rng, n, -149, 127), random_floats(rng, n, -149, 127))
