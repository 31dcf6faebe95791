"""g(r) of subroutine g (g.f:22-144) on the CPU: the oracle's pair histogram
against a numpy restatement of the same arithmetic (bin for bin), and the
normalization of yukawamd_b200.gofr on an ideal gas, where g(r) ~ 1."""
import numpy as np

from oracle.oracle import Oracle
from yukawamd_b200 import configs
from yukawamd_b200.gofr import GofR, write


def numpy_counts(x, xl, nbin):
    x = x.reshape(-1, 3)
    n = len(x)
    xlmin = min(xl)
    fac2 = float(np.float32(np.float32(2.0) * np.float32(nbin) / np.sqrt(np.float32(3.0)))) / xlmin
    tiny = float(np.float32(1.e-15))
    counts = np.zeros(nbin)
    for i in range(n - 1):
        yy = np.abs(x[i] - x[i + 1:])
        yy = np.minimum(yy, np.array(xl) - yy)
        rr = ((yy[:, 0] * yy[:, 0] + yy[:, 1] * yy[:, 1]) + yy[:, 2] * yy[:, 2])
        rr = np.sqrt(rr) + tiny
        ii = np.minimum(nbin, (fac2 * rr + 1.0).astype(np.int64))
        np.add.at(counts, ii - 1, 1.0)
    return counts


def test_oracle_counts_equal_numpy():
    w = configs.pure_ion_ocp(5, 400)
    p = w.yk_params()
    for nbin in (7, 64, 1000):
        c = Oracle("double").gofr_counts(p, w.x, nbin)
        assert np.array_equal(c, numpy_counts(w.x, list(p.xl), nbin))
        assert c.sum() == 400 * 399 / 2


class _FakeEngine:
    def __init__(self, orc, p, x):
        self.orc, self.p, self.x = orc, p, x

    def gofr_counts(self, nbin, counts):
        counts += self.orc.gofr_counts(self.p, self.x, nbin)
        return counts


def test_ideal_gas_is_flat(tmp_path):
    rng = np.random.default_rng(7)
    n, L = 3000, 50.0
    w = configs.pure_ion_ocp(6, 8)
    p = w.yk_params()
    for k in range(3):
        p.xl[k] = L
    orc = Oracle("double", threads=4)
    g = GofR(nbin=20, ngroup=2)
    for ig in (1, 2):
        x = rng.uniform(0.0, L, size=3 * n)
        g.take(_FakeEngine(orc, p, x), ig)
    rr, gm, gs = g.finish(n, n / L ** 3, [L, L, L])
    mid = (rr > 5.0) & (rr < 0.45 * L)          # away from r = 0 and the corner bins
    assert np.all(np.abs(gm[mid] - 1.0) < 0.05)
    assert np.all(gs >= 0.0)
    write(tmp_path / "g.out", rr, gm, gs)
    line = open(tmp_path / "g.out").readline()
    assert len(line.rstrip("\n")) == 15 + 2 + 15 + 2 + 15


def test_sofq_of_ideal_gas_is_one():
    """S(q) of s.f on g = 1 everywhere is 1 for every q, and for a g with one
    extra bump it follows the transform's formula term by term."""
    g = GofR(nbin=40, ngroup=2)
    g.gnorm = np.ones((40, 2))
    q, sm, ss = g.sofq(1000, 0.05, [30.0, 30.0, 30.0], 0.2, 0.1, 12)
    assert np.allclose(q, 0.2 + 0.1 * np.arange(12))
    assert np.all(sm == 1.0) and np.all(ss == 0.0)
    g.gnorm[5, :] = 2.0
    q, sm, _ = g.sofq(1000, 0.05, [30.0, 30.0, 30.0], 0.2, 0.1, 3)
    dd = 30.0 / 40 * float(np.float32(np.sqrt(3.0))) / 2
    r5 = (6 - 0.5) * dd
    want = 4 * np.pi * dd * 0.05 * r5 ** 2 * np.sin(q * r5) / (q * r5) + 1
    assert np.allclose(sm, want, rtol=1e-12)
