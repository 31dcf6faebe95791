"""Test helpers for the run driver.

`md_reference` restates md.F:63-205 one step at a time over the oracle
(accel, newton, ttot, tnorm, cancel_vcom, strain as the reference calls them);
`OracleEngine` is the engine interface the driver uses (accel, run, ttot,
tnorm, cancel_vcom, strain), carried out by the same oracle calls.  Running
yukawamd_b200.driver.run_md over OracleEngine must reproduce md_reference bit
for bit: that checks the driver's call planning on the CPU.
"""
import math

import numpy as np

from yukawamd_b200 import abi
from yukawamd_b200.driver import XNOSTRAIN, f_float, mdmod


def _pp6(s):
    p = s.pp
    return (p[0], p[3], p[6], p[4], p[7], p[8])


def _statt(xa, xa2, n, xave, x2ave):
    xa = xa / f_float(n)
    xa2 = xa2 / f_float(n)
    dx = math.sqrt(abs(xa2 - xa * xa) / f_float(n - 1)) if n > 1 else 0.0
    return xa, dx, xave + xa, x2ave + xa * xa


class OracleEngine:
    def __init__(self, orc, params, x, v, zii, aii):
        self.orc = orc
        self.params = params
        self.x, self.v = x.copy(), v.copy()
        self.vold = np.zeros_like(self.v)
        self.zii, self.aii = zii, aii
        self.n = len(aii)
        self.a = np.zeros(3 * (self.n + 3))
        self.time = params.time
        self.xl0 = None

    def accel(self, meas):
        a, s = self.orc.accel(self.params, self.x, self.zii, self.aii, meas)
        self.a[:] = a
        s.time = self.time
        return s

    def newton(self, meas):
        s = self.orc.newton(self.params, self.x, self.v, self.vold, self.a, self.zii, self.aii, meas)
        self.time = self.time + self.params.dt
        s.time = self.time
        return s

    def run(self, k, m, series=True):
        buf = (abi.YkScalars * k)()
        for j in range(k):
            buf[j] = self.newton(m > 0 and (j + 1) % m == 0)
        return buf

    def ttot(self):
        return self.orc.ttot(self.params, self.v, self.aii)

    def tnorm(self):
        self.orc.tnorm(self.params, self.v, self.aii)

    def cancel_vcom(self):
        self.orc.cancel_vcom(self.params, self.v, self.aii)

    def strain(self, deps, xl0):
        xl = np.array(list(self.params.xl), dtype=float)
        self.orc.strain(self.params, self.x, xl, np.array(xl0, float), np.array(deps, float))
        for k in range(3):
            self.params.xl[k] = xl[k]
        return list(xl)


def md_reference(eng, ctl):
    """md.F:63-205, one call at a time, on an OracleEngine.  Returns a dict
    with the same records as driver.MDResult."""
    out = dict(warmup=[], e_lines=[], p_lines=[], meas=[], groups=[], ckpt=[])
    xl0 = list(ctl.xl0) if ctl.xl0 is not None else list(eng.params.xl)
    deps = ctl.deps
    s = eng.accel(True)
    ek = eng.ttot()
    out["initial"] = dict(ev=s.ev, ek=ek, e=s.ev + ek, px=s.px)
    istep = 0
    for _ in range(ctl.nwgroup):
        for _ in range(ctl.nwsteps):
            eng.newton(False)
            istep += 1
            if mdmod(istep, ctl.nckpt) == 0:
                out["ckpt"].append((istep, eng.time))
        eng.cancel_vcom()
        eng.tnorm()
        out["warmup"].append((istep, eng.time))
    if istep > 0 and mdmod(istep, ctl.nckpt) != 0:
        out["ckpt"].append((istep, eng.time))
    evave = ev2ave = pave = p2ave = 0.0
    istep = 0
    for ig in range(1, ctl.ngroup + 1):
        eva = ev2a = pa = p2a = 0.0
        for _ in range(ctl.ntot * ctl.nind):
            if mdmod(istep, ctl.ncom) == 0:
                eng.cancel_vcom()
            if mdmod(istep, ctl.ntnorm) == 0:
                eng.tnorm()
            eng.strain(deps, xl0)
            dm = mdmod(istep + 1, ctl.nind) == 0 or mdmod(istep + 1, ctl.nptensor) == 0
            s = eng.newton(dm)
            istep += 1
            if mdmod(istep, ctl.nind) == 0:
                eva += s.ev
                ev2a += s.ev ** 2
                pa += s.px
                p2a += s.px ** 2
                out["e_lines"].append((istep, s.time, s.ev, s.ek, s.ek + s.ev, s.px))
            if mdmod(istep, ctl.nptensor) == 0:
                out["p_lines"].append((istep, s.time) + _pp6(s))
            if dm:
                out["meas"].append((istep, s.time, s.ev, s.ek, s.px) + _pp6(s))
            if mdmod(istep, ctl.nckpt) == 0:
                out["ckpt"].append((istep, eng.time))
        eva, dev, evave, ev2ave = _statt(eva, ev2a, ctl.ntot, evave, ev2ave)
        pa, dp, pave, p2ave = _statt(pa, p2a, ctl.ntot, pave, p2ave)
        out["groups"].append((ig, eng.time, eva, dev, pa, dp))
    if ctl.ngroup > 0:
        out["evave"], out["devave"], _, _ = _statt(evave, ev2ave, ctl.ngroup, 0.0, 0.0)
        out["pave"], out["dpave"], _, _ = _statt(pave, p2ave, ctl.ngroup, 0.0, 0.0)
    if istep > 0 and mdmod(istep, ctl.nckpt) != 0:
        out["ckpt"].append((istep, eng.time))
    s = eng.accel(True)
    ek = eng.ttot()
    out["final"] = dict(ev=s.ev, ek=ek, e=s.ev + ek, px=s.px, xl=list(eng.params.xl))
    return out


__all__ = ["OracleEngine", "md_reference", "XNOSTRAIN"]
