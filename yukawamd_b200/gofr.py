"""The two-particle correlation function g(r) of subroutine g (g.f:22-144).

The reference keeps the routine but comments out its calls (md.F:64, 154,
184-186): it is "not ready for use" by its own note (g.f:11-14) and treats
every particle as one species.  `GofR` restates its three phases:

  ig = 0    allocate and zero the histogram of every measurement group (g.f:43-48)
  ig > 0    add the pair-distance histogram of the current configuration
            (g.f:55-71) -- on the GPU, Engine.gofr_counts (yk_gofr_counts)
  ig = -1   normalize by the ideal-gas shell counts and average over the
            groups (g.f:97-130), with the reference's REAL*4 promotions

and `write` prints the g.out lines (format 10000: f15.8, 2x, es15.8, 2x, es15.8).
`GofR.sofq` is subroutine s (s.f:22-97), which md.F would call between g(-1)
and g(-2): the static structure factor S(q) = 1 + rho 4 pi int r^2
sin(qr)/(qr) (g(r) - 1) dr on the normalized g of every group.
"""
import math

import numpy as np

PI = 3.14159265358979324     # md_globals.f:28


def _f32(v):
    return float(np.float32(v))


class GofR:
    def __init__(self, nbin, ngroup):
        """ig = 0 (g.f:43-48)."""
        self.nbin = int(nbin)
        self.ngroup = int(ngroup)
        self.gg = np.zeros((self.nbin, self.ngroup))
        self.cgg = np.zeros(self.ngroup)

    def take(self, engine, ig):
        """ig > 0 (g.f:51-71): one configuration into group ig (1-based)."""
        counts = np.ascontiguousarray(self.gg[:, ig - 1])
        engine.gofr_counts(self.nbin, counts)
        self.gg[:, ig - 1] = counts
        self.cgg[ig - 1] += 1

    def finish(self, n, rho, xl):
        """ig = -1 (g.f:97-130).  Returns (rr, gmean, gstd) per bin."""
        nbin, ngroup = self.nbin, self.ngroup
        ngspec = n                                            # g.f:98-101: every particle
        xlmin = min(xl)
        dd = xlmin / _f32(nbin) * _f32(math.sqrt(3.0)) / 2.0  # sqrt(3.) is REAL*4
        fac = _f32(n) / (_f32(_f32(ngspec) ** 2) * rho * dd * 2.0 * PI)
        g = np.empty((nbin, ngroup))
        rr = np.empty(nbin)
        for j in range(1, nbin + 1):
            rr[j - 1] = _f32(j - 0.5) * dd                    # (j-.5) is REAL*4
            for i in range(ngroup):
                g[j - 1, i] = fac * self.gg[j - 1, i] / (self.cgg[i] + _f32(1.e-30)) / rr[j - 1] ** 2
        self.gnorm = g                                       # gg(:,:,0) after g.f:106-111
        gmean = np.empty(nbin)
        gstd = np.empty(nbin)
        for j in range(nbin):
            m = 0.0
            m2 = 0.0
            for i in range(ngroup):
                m += g[j, i]
                m2 += g[j, i] ** 2
            m = m / _f32(ngroup)
            m2 = m2 / _f32(ngroup)
            gmean[j] = m
            gstd[j] = math.sqrt(abs(m2 - m ** 2) / ngroup)
        return rr, gmean, gstd

    def sofq(self, n, rho, xl, qmin, dq, nsbin):
        """s.f:22-97 on the groups normalized by finish().  Returns (q, smean, sstd)."""
        nbin, ngroup = self.nbin, self.ngroup
        nbmax = int(_f32(nbin / _f32(math.sqrt(3.0))))         # integer = REAL*4 quotient
        xlmin = min(xl)
        dd = xlmin / _f32(nbin) * _f32(math.sqrt(3.0)) / 2
        ngspec = n
        rhox = _f32(_f32(ngspec) / _f32(n)) * rho
        r = [(_f32(k) - _f32(0.5)) * dd for k in range(1, nbmax + 1)]
        ss = np.empty((nsbin, ngroup))
        for i in range(ngroup):
            q = qmin - dq
            for j in range(nsbin):
                q = q + dq
                acc = 0.0
                for k in range(nbmax):
                    rq = q * r[k]
                    acc = acc + (r[k] ** 2) * (math.sin(rq) / rq) * (self.gnorm[k, i] - 1.0)
                ss[j, i] = 4.0 * PI * dd * rhox * acc + 1.0
        qs = np.empty(nsbin)
        smean = np.empty(nsbin)
        sstd = np.empty(nsbin)
        q = qmin - dq
        for j in range(nsbin):
            q = q + dq
            m = 0.0
            m2 = 0.0
            for i in range(ngroup):
                m += ss[j, i]
                m2 += ss[j, i] ** 2
            m = m / _f32(ngroup)
            m2 = m2 / _f32(ngroup)
            qs[j] = q
            smean[j] = m
            sstd[j] = math.sqrt(abs(m2 - m ** 2) / _f32(ngroup))
        return qs, smean, sstd


def write(path, rr, gmean, gstd):
    """g.out lines of g.f:126 (format 10000); also the s.out lines of s.f:86."""
    with open(path, "w") as f:
        for a, b, c in zip(rr, gmean, gstd):
            f.write("%15.8f  %15.8E  %15.8E\n" % (a, b, c))
