"""The mixed form's ion displacement from the FP32 shadow's hi/lo parts
(store_shadow and screen_d_x2 in yukawamd_b200/csrc/yk_force.cuh), restated
in numpy float32 arithmetic.

store_shadow keeps every coordinate as hi = x rounded to the grid of
SHADOW_Q fm and lo = x - hi rounded to FP32.  On that grid every value below
SHADOW_EXACT = 2^24 SHADOW_Q is an FP32 number, so

  dc = fl(xh_j - xh_i)            is exact,
  d1 = fl(dc - k Lh), k in {-1, 0, 1}, Lh the box on the grid, is exact,

and the displacement d = d1 + ((xl_j - xl_i) - k Ll) carries one rounding of
its own.  The tests check those exactness claims and that -d is within 1e-7
relative of the reference's FP64 conditional minimum image x_i - x_j
(int_ion_pure.f:147-152) for pairs away from |d| = L/2 (the kernel takes this
path only when every interacting pair is, fa.img_k), including pairs that
straddle the periodic boundary, for boxes from 30 fm to near the 16,384 fm
limit of the path (fa.lo).
"""
import os
import re

import numpy as np
import pytest

F32 = np.float32
SRC = os.path.join(os.path.dirname(__file__), "..", "yukawamd_b200", "csrc", "yk_force.cuh")


def source_constants():
    text = open(SRC).read()
    q = re.search(r"constexpr double SHADOW_Q = 1\.0 / ([0-9.]+);", text)
    exact = re.search(r"constexpr double SHADOW_EXACT = ([0-9.]+);", text)
    return 1.0 / float(q.group(1)), float(exact.group(1))


Q, EXACT = source_constants()


def hi_part(x):
    return np.rint(x / Q) * Q


def fma32(a, b, c):
    """float32 fused multiply-add where a*b + c is exact in float64."""
    return (a.astype(np.float64) * b.astype(np.float64) + c.astype(np.float64)).astype(F32)


def test_grid_constants():
    assert EXACT == 2.0 ** 24 * Q
    assert Q == 2.0 ** round(np.log2(Q))


def pairs(L, n, rng):
    xi = rng.uniform(0.0, L, n)
    xj = rng.uniform(0.0, L, n)
    # half of the pairs close together, many of them across the boundary
    m = n // 2
    xj[:m] = np.mod(xi[:m] + rng.normal(0.0, 3.0, m), L)
    return xi, xj


@pytest.mark.parametrize("L", [30.0, 100.794, 384.957, 916.621, 8000.0, 16000.0])
def test_displacement_from_hi_lo(L):
    rng = np.random.default_rng(int(L))
    xi, xj = pairs(L, 200000, rng)
    hi_i, hi_j = hi_part(xi), hi_part(xj)
    fhi_i, fhi_j = hi_i.astype(F32), hi_j.astype(F32)
    assert np.array_equal(fhi_i.astype(np.float64), hi_i)          # hi parts are FP32 numbers
    lo_i, lo_j = (xi - hi_i).astype(F32), (xj - hi_j).astype(F32)
    assert np.all(np.abs(lo_i) <= Q / 2)
    Lh = F32(hi_part(L))
    Ll = F32(L - hi_part(L))
    invL = F32(1.0 / L)
    MAG = F32(12582912.0)

    dc = (fhi_j + (-fhi_i)).astype(F32)
    assert np.array_equal(dc.astype(np.float64), hi_j - hi_i)       # exact
    k = (fma32(dc, np.full_like(dc, invL), np.full_like(dc, MAG)) + F32(-MAG)).astype(F32)
    assert set(np.unique(k)) <= {F32(-1.0), F32(0.0), F32(1.0)}
    d1 = fma32(np.full_like(dc, -Lh), k, dc)
    assert np.array_equal(d1.astype(np.float64), dc.astype(np.float64) - float(Lh) * k)   # exact
    e = fma32(np.full_like(dc, -Ll), k, (lo_j + (-lo_i)).astype(F32))
    d = (d1 + e).astype(F32)

    ref = xi - xj                                                   # int_ion_pure.f:147-152
    ref = np.where(ref > L / 2, ref - L, np.where(ref < -L / 2, ref + L, ref))
    away = np.abs(ref) < 0.49 * L
    err = np.abs(-d.astype(np.float64) - ref)[away]
    rel = err / np.maximum(np.abs(ref[away]), 1e-3)
    assert rel.max() < 1.0e-7
    # the FP32 cast of the exact displacement, for scale
    cast = np.abs(ref.astype(F32).astype(np.float64) - ref)[away] / np.maximum(np.abs(ref[away]), 1e-3)
    assert rel.max() < 2.0 * cast.max()
