"""The FP32 form rebuilds its (rcut + skin) neighbour lists with a cheap test:
FP32 arithmetic on the top 16 bits of each 32-bit fixed-point centre
difference, against rcut + skin widened by sqrt(3) L_max 2^-16 and a relative
1e-5 (kernels.cu, build_lists).  The lists only have to contain every pair
within rcut + skin, so the test must never reject such a pair.  This restates
it in numpy (float32, the same operation order) and checks that on pairs
placed at and around the boundary, in boxes of 10-120 A.  The device may fuse
the squares into FMAs (a rounding difference near 1e-7 relative); the margin
between rcut + skin and the widened bound is at least 1e-5 relative, so the
property holds for either rounding."""
import numpy as np
import pytest


def fixed(r):
    # box fraction in [0, 1) -> (r - 1/2) 2^32 as a wrapping int32 (fix_coord)
    return ((np.rint((r - 0.5) * 2.0 ** 32).astype(np.int64) + 2 ** 31) % 2 ** 32 - 2 ** 31).astype(np.int32)


def wrap_diff(a, b):
    return ((a.astype(np.int64) - b.astype(np.int64) + 2 ** 31) % 2 ** 32 - 2 ** 31).astype(np.int32)


def cheap_keep(wd, L, rl):
    lsc = (L / 65536.0).astype(np.float32)
    hx = (wd >> 16).astype(np.int32)
    f = (hx.astype(np.float32) * lsc).astype(np.float32)   # the bit trick converts hx exactly
    r2 = (f[:, 0] * f[:, 0] + f[:, 1] * f[:, 1]).astype(np.float32) + (f[:, 2] * f[:, 2]).astype(np.float32)
    rw = (rl + np.sqrt(3.0) * L.max() / 65536.0) * (1.0 + 1e-5)
    return r2.astype(np.float32) < np.float32(rw * rw)


@pytest.mark.parametrize("L", [(10.0, 10.0, 10.0), (25.0, 25.0, 60.0), (120.0, 118.0, 30.0)])
def test_cheap_rebuild_test_keeps_every_pair_within_rcut_plus_skin(L):
    rng = np.random.default_rng(7)
    L = np.array(L)
    rl = min(0.49 * L.min(), 9.9)
    n = 200000
    ri = rng.random((n, 3))
    # partners at distances concentrated around rl (inside and just outside)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    dist = rl * (1.0 + rng.uniform(-2e-4, 2e-4, n))
    rj = (ri + d * dist[:, None] / L) % 1.0
    a, b = fixed(ri), fixed(rj)
    wd = wrap_diff(a, b)
    exact = ((wd.astype(np.float64) / 2.0 ** 32 * L) ** 2).sum(axis=1) < rl * rl
    kept = cheap_keep(wd, L, rl)
    assert exact.any() and (~exact).any()
    assert not np.any(exact & ~kept)           # nothing within rcut + skin is dropped
    # and the widening stays small: what is kept lies within rl (1 + 1e-4)
    far = ((wd.astype(np.float64) / 2.0 ** 32 * L) ** 2).sum(axis=1) > (rl * (1 + 1e-4 + 2e-5 * L.max())) ** 2
    assert not np.any(kept & far)
