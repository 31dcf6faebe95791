"""The mixed form's FP32 exp(-t) (exp_neg_f32 in yukawamd_b200/csrc/yk_common.cuh).

1. The degree-6 polynomial for 2^f on [-1/2, 1/2] with the source's float32
   constants is within 2e-8 (0.3 ulp) relative of 2^f; a fresh fit of the
   same form (relative-error least squares with Lawson reweighting on 4001
   Chebyshev nodes) reaches 2.5e-9 in exact arithmetic, so the degree leaves
   the error to the float32 rounding.  (High-order coefficients of such fits
   are ill-conditioned, so they are not compared one by one.)
2. A float32 restatement of the device function (magic-number rounding, the
   Cody-Waite split of t*log2(e), Horner with fused multiply-adds, exponent
   scaling through the bits) stays within 2 ulp of exp(-t) for t in [0, 80],
   which covers every argument of the pair terms (mu r <= mu r_c, and
   r^2 / (2 Lambda) <= rncut^2 / (2 Lambda) = 53 for the default HPP cutoff).
"""
import re
import os

import numpy as np

SRC = os.path.join(os.path.dirname(__file__), "..", "yukawamd_b200", "csrc", "yk_common.cuh")


def source_coefficients():
    text = open(SRC).read()
    body = text[text.index("float exp_neg_f32"):]
    body = body[:body.index("}")]
    first = float(re.search(r"float p = ([0-9.eE+-]+)f;", body).group(1))
    rest = [float(c) for c in re.findall(r"p = fmaf\(p, f, ([0-9.eE+-]+)f\);", body)]
    return [first] + rest          # highest degree first


def lawson_fit(deg=6, nodes=4001, iters=60):
    k = np.arange(nodes)
    x = 0.5 * np.cos(np.pi * (k + 0.5) / nodes)
    y = np.exp2(x)
    V = np.vander(x, deg + 1)                  # highest degree first
    w = np.ones(nodes)
    for _ in range(iters):
        A = V * (w / y)[:, None]
        c, *_ = np.linalg.lstsq(A, w, rcond=None)
        e = np.abs(V @ c / y - 1.0)
        w = w * e
        w = w / w.sum() * nodes
    return c, np.max(np.abs(V @ c / y - 1.0))


def test_coefficients_are_the_fit():
    c_src = np.array(source_coefficients())
    assert len(c_src) == 7
    _c_fit, err = lawson_fit()
    assert err < 2.5e-9
    x = np.linspace(-0.5, 0.5, 20001)
    p_src = np.polyval(c_src, x)
    assert np.max(np.abs(p_src / np.exp2(x) - 1.0)) < 2e-8


def _fma32(a, b, c):
    # the exact product of two floats fits a double; one rounding to float32
    return np.float32(np.float64(a) * np.float64(b) + np.float64(c))


def exp_neg_f32(t):
    f32 = np.float32
    L2E_HI = f32(1.44269502162933349609375)
    L2E_LO = f32(1.925963033500011079e-8)
    MAGIC = f32(12582912.0)
    t = f32(t)
    yh = f32(-t * L2E_HI)
    yl = _fma32(-t, L2E_HI, -yh)
    yl = _fma32(-t, L2E_LO, yl)
    kb = f32(yh + MAGIC)
    k = f32(kb - MAGIC)
    f = f32(f32(yh - k) + yl)
    c = source_coefficients()
    p = f32(c[0])
    for cm in c[1:]:
        p = _fma32(p, f, f32(cm))
    ki = int(np.array(kb, dtype=np.float32).view(np.int32)) - 0x4B400000
    if k < -125.0:
        return f32(0.0)
    bits = int(np.array(p, dtype=np.float32).view(np.int32)) + (ki << 23)
    return np.array(bits, dtype=np.int32).view(np.float32).item()


def test_restated_exp_within_two_ulp():
    rng = np.random.default_rng(3)
    ts = np.concatenate([np.linspace(0.0, 80.0, 801), rng.uniform(0.0, 20.0, 600),
                         [0.0, 1e-8, 0.5, 0.6931472, 1.0, 10.0, 53.0, 80.0]])
    worst = 0.0
    for t in ts:
        got = exp_neg_f32(t)
        ref = np.exp(-np.float64(np.float32(t)))
        ulp = np.spacing(np.float32(ref))
        worst = max(worst, abs(got - ref) / ulp)
    assert worst <= 2.0, worst


def test_underflow_flushes_to_zero():
    assert exp_neg_f32(100.0) == 0.0
    assert exp_neg_f32(1e5) == 0.0


# ---- FP64 exp(-t) (exp_neg_f64, table-driven) ------------------------------

def _f64_source_table():
    text = open(SRC).read()
    body = text[text.index("g_exp2_256[256] = {"):]
    body = body[body.index("{") + 1:body.index("};")]
    return [float(v) for v in body.replace("\n", " ").split(",") if v.strip()]


def _fma64(a, b, c):
    from fractions import Fraction
    return float(Fraction(a) * Fraction(b) + Fraction(c))   # one rounding


def exp_neg_f64(t):
    import struct
    tab = _f64_source_table()
    MAG = 6755399441055744.0
    kd = _fma64(-t, 369.3299304675746, MAG)
    nf = kd - MAG
    r = _fma64(-nf, 9.058776616587108e-20, _fma64(-nf, 0.0027076061740622863, -t))
    q = 1.0 / 24.0
    for c in (1.0 / 6.0, 0.5, 1.0):
        q = _fma64(q, r, c)
    p = q * r
    bits = struct.unpack("<q", struct.pack("<d", kd))[0]
    ni = ((bits & 0xffffffff) ^ 0x80000000) - 0x80000000      # low word as int32
    tj = tab[ni & 255]
    res = _fma64(tj, p, tj)
    rb = struct.unpack("<q", struct.pack("<d", res))[0]
    rb += (ni >> 8) << 52
    return 0.0 if t > 700.0 else struct.unpack("<d", struct.pack("<q", rb))[0]


def test_f64_table_is_correctly_rounded():
    from decimal import Decimal, getcontext
    getcontext().prec = 50
    ln2 = Decimal(2).ln()
    tab = _f64_source_table()
    assert len(tab) == 256
    for j, v in enumerate(tab):
        assert v == float((Decimal(j) / 256 * ln2).exp())


def test_f64_exp_within_three_ulp():
    from decimal import Decimal, getcontext
    getcontext().prec = 50
    rng = np.random.default_rng(11)
    ts = np.concatenate([[0.0, 1e-300, 1e-9, 0.5, 1.0, np.log(2.0) / 512, np.log(2.0) / 128, 10.0, 53.0, 699.0],
                         rng.uniform(0.0, 12.0, 300), rng.uniform(0.0, 700.0, 100)])
    worst = 0.0
    for t in ts:
        t = float(t)
        got = exp_neg_f64(t)
        ref = (-Decimal(t)).exp()
        worst = max(worst, float(abs(Decimal(got) - ref) / Decimal(float(np.spacing(float(ref))))))
    assert worst <= 3.0, worst
    assert exp_neg_f64(701.0) == 0.0


def test_rsqrt_second_order_error_bound():
    """rsqrt_nr64 (yukawamd_b200/csrc/yk_common.cuh): one second-order
    correction y + y e (1/2 + 3e/8), e = fma(-(x y), y, 1), of an FP32
    estimate y.  Restated with each FMA rounded once (exact rational
    arithmetic, then one rounding to double) and the estimate off by up to
    2^-21 relative either way (the hardware's is within about 2^-22), over
    r^2 from 1e-4 to 1e9: the result is within 1 ulp of 1/sqrt(x) (computed
    to 50 digits)."""
    from decimal import Decimal, getcontext
    from fractions import Fraction
    getcontext().prec = 50

    def fma(a, b, c):
        return float(Fraction(a) * Fraction(b) + Fraction(c))

    rng = np.random.default_rng(11)
    xs = np.concatenate([10.0 ** rng.uniform(-4, 9, 400), [1.0, 2.0, 0.25, 8.9e4, 1e9]])
    worst = 0.0
    for x in xs:
        x = float(x)
        exact = float(1 / Decimal(x).sqrt())
        for rel in (-2.0 ** -21, 0.0, 2.0 ** -21, rng.uniform(-2.0 ** -21, 2.0 ** -21)):
            y = float(np.float32(exact * (1.0 + rel)))
            e = fma(-(x * y), y, 1.0)
            r = fma(y * e, fma(e, 0.375, 0.5), y)
            worst = max(worst, abs(r - exact) / np.spacing(exact))
    assert worst <= 1.0, worst


def test_far_mask_rounds_the_pair_term_to_zero():
    """ion_terms_x2 and coulomb_terms_x2 (yukawamd_b200/csrc/yk_force.cuh)
    give a masked pair r^2 = 1e36 instead of multiplying its term by the
    mask.  Restated in numpy float32 with the reciprocal-root estimate off by
    up to 2^-21 either way: 1/r and 1/r^2 stay normal, mu r stays finite, and
    q = prefactor e^{-mu r} (1/r)^3 is exactly 0 for every mu >= 0 (mu = 0,
    unscreened, included) and prefactors up to 1e6, so fs = mu r q + q = 0."""
    f32 = np.float32
    r2s = f32(1e36)
    for rel in (-2.0 ** -21, 0.0, 2.0 ** -21):
        rinv = f32(f32(1.0 / np.sqrt(1e36)) * f32(1.0 + rel))
        rr = f32(rinv * rinv)
        assert rr >= np.finfo(np.float32).tiny
        for mu in (0.0, 1e-3, 0.1, 10.0):
            mr = f32(f32(mu) * f32(r2s * rinv))
            assert np.isfinite(mr)
            e = f32(np.exp2(np.float64(mr) * -1.4426950408889634))   # 0 unless mu = 0
            for pre in (1.0, 1.44, 1e6):
                er = f32(f32(e * rinv) * f32(pre))
                q = f32(er * rr)
                assert q == 0.0, (rel, mu, pre, q)
                assert f32(mr * q + q) == 0.0
