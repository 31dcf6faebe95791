"""The reference's run driver (md.F:63-205) over the device engine.

`run_md(engine, ctl)` takes the run-control integers of md_globals.f:73-86
(nwgroup, nwsteps, ngroup, ntot, nind, nptensor, ncom, ntnorm, nckpt, nout)
and the strain rates deps (md_globals.f:62) and makes, in the reference's
order, every call md.F makes:

  accel(.true.), ttot                                   md.F:69-70
  warm-up: nwgroup x (nwsteps x newton(.false.),
           cancel_vcom, tnorm)                          md.F:87-101
  measurement: per step cancel_vcom if mdmod(istep,ncom)=0,
           tnorm if mdmod(istep,ntnorm)=0, strain,
           newton(do_measurements)                      md.F:125-130
  records: 'e' lines every nind steps, 'p' lines every nptensor steps,
           the .meas records on measuring steps, the block statistics of
           statt per group and over groups               md.F:131-172
  final accel(.true.), ttot, stretch, density           md.F:188-200

and checkpoints / configuration saves through caller hooks (md.F:93,
md.F:156-157, md.F:103, md.F:173).

Everything runs on the device state.  Between host passes the steps go to
yk_run as CUDA graphs: `plan` cuts each stretch into yk_run calls whose
measurement pattern is exactly the reference's do_measurements.  A pass that
md.F makes every step (strain with a strain rate set) makes every step its
own call.  Without a strain rate, strain only re-wraps x > xl (strain.f:73-79),
which is a no-op after a Verlet step: the integrators already leave every
coordinate at or below xl (vel_verlet_2.f:39-40), so the driver runs that
re-wrap once, before the first measurement step, and not again.
"""
from dataclasses import dataclass, field
import math

import numpy as np

XNOSTRAIN = 1000.0          # md_globals.f: a strain rate that means "none"


def mdmod(p, q):
    """md.F:248-256: mod(p, q), or -1 when q = 0 (q = 0 means "never")."""
    return -1 if q == 0 else p % q


def f_float(i):
    """Fortran float() of an integer: a default-REAL (f32) value."""
    return float(np.float32(i))


def measures(istep1, nind, nptensor):
    """do_measurements for the step that ends at istep1 (md.F:129)."""
    return mdmod(istep1, nind) == 0 or mdmod(istep1, nptensor) == 0


def plan(s0, s1, nind, nptensor):
    """yk_run calls (nsteps, meas_every) that advance from istep s0 to s1 with
    step istep measuring exactly when measures(istep + 1).  A call (k, m)
    measures its steps s = m, 2m, ... (1-based within the call)."""
    calls = []
    last = s0
    for istep in range(s0, s1):
        if measures(istep + 1, nind, nptensor):
            k = istep + 1 - last
            if calls and calls[-1][1] == k and calls[-1][0] % k == 0:
                calls[-1] = (calls[-1][0] + k, k)
            else:
                calls.append((k, k))
            last = istep + 1
    if last < s1:
        r = s1 - last
        if calls and calls[-1][1] > r:
            calls[-1] = (calls[-1][0] + r, calls[-1][1])     # no multiple of m in the tail
        else:
            calls.append((r, 0))
    return calls


def statt(xa, xa2, n, xave, x2ave):
    """md.F:227-240.  Returns (xa, xa2, dx, xave, x2ave) after the update."""
    xa = xa / f_float(n)
    xa2 = xa2 / f_float(n)
    dx = math.sqrt(abs(xa2 - xa * xa) / f_float(n - 1)) if n > 1 else 0.0
    return xa, xa2, dx, xave + xa, x2ave + xa * xa


def strain_edges(xl, xl0, deps, dt):
    """strain.f:31-69: the new edge lengths for one step (host arithmetic)."""
    xl = list(xl)
    on = [deps[k] != XNOSTRAIN for k in range(3)]
    sel = on[0] * 1 + on[1] * 2 + on[2] * 4
    for k in range(3):
        if on[k]:
            xl[k] = xl[k] + deps[k] * dt * xl0[k]
    if sel in (1, 2, 4):
        k = {1: 0, 2: 1, 4: 2}[sel]
        for j in range(3):
            if j != k:
                xl[j] = xl0[j] * math.sqrt(xl0[k] / xl[k])
    elif sel in (3, 5, 6):
        j = {3: 2, 5: 1, 6: 0}[sel]
        a, b = [t for t in range(3) if t != j]
        xl[j] = xl0[j] * (xl0[a] / xl[a]) * (xl0[b] / xl[b])
    return xl


@dataclass
class RunControl:
    """md_globals.f:73-86 (0 = never) plus the strain rates."""
    nwgroup: int = 0
    nwsteps: int = 0
    ngroup: int = 0
    ntot: int = 0
    nind: int = 0
    nptensor: int = 0
    ncom: int = 0
    ntnorm: int = 0
    nckpt: int = 0
    nout: int = 0
    deps: tuple = (XNOSTRAIN, XNOSTRAIN, XNOSTRAIN)
    xl0: tuple = None                 # gage dimensions; default the initial xl

    @property
    def strained(self):
        return any(d != XNOSTRAIN for d in self.deps)


@dataclass
class MDResult:
    initial: dict = None                              # ev, ek, e, px
    warmup: list = field(default_factory=list)        # (istep, time)
    e_lines: list = field(default_factory=list)       # (istep, time, ev, ek, e, px)
    p_lines: list = field(default_factory=list)       # (istep, time, pxx, pxy, pxz, pyy, pyz, pzz)
    meas: list = field(default_factory=list)          # .meas: (istep, time, ev, ek, px, 6 x pp)
    groups: list = field(default_factory=list)        # (ig, time, eva, dev, pa, dp)
    evave: float = 0.0
    devave: float = 0.0
    pave: float = 0.0
    dpave: float = 0.0
    final: dict = None                                # xl, stretch, rho, ev, ek, e, px
    calls: int = 0                                    # yk_run / yk_newton calls made


def _pp6(s):
    p = s.pp
    return (p[0], p[3], p[6], p[4], p[7], p[8])       # pp(1,1) pp(1,2) pp(1,3) pp(2,2) pp(2,3) pp(3,3)


class _State:
    """The driver's copies of the reference globals it reads."""

    def __init__(self, engine):
        self.e = engine
        self.time = engine.params.time
        self.last = None            # yk_scalars of the latest step (ev, ek, px, pp globals)


def run_md(engine, ctl, on_checkpoint=None, on_save=None):
    """Run md.F's warm-up and measurement phases on `engine` (an Engine whose
    params carry dt, kT, xl ...).  on_checkpoint(engine, istep, time, scalars)
    and on_save(engine, istep, time, scalars) are called where md.F calls
    checkpoint and save_config.  Returns an MDResult."""
    st = _State(engine)
    res = MDResult()
    dt = engine.params.dt
    xl0 = list(ctl.xl0) if ctl.xl0 is not None else list(engine.params.xl)
    n = engine.n

    def ckpt(istep):
        if on_checkpoint is not None:
            on_checkpoint(engine, istep, st.time, st.last)

    s = engine.accel(True)                                   # md.F:69
    ek = engine.ttot()                                       # md.F:70
    st.last = s
    res.initial = dict(ev=s.ev, ek=ek, e=s.ev + ek, px=s.px)

    # -- warm-up (md.F:87-103) --------------------------------------------
    istep = 0
    for _ in range(ctl.nwgroup):
        done = 0
        while done < ctl.nwsteps:
            k = ctl.nwsteps - done
            if ctl.nckpt > 0:
                k = min(k, ctl.nckpt - istep % ctl.nckpt)
            ser = engine.run(k, 0, series=True)
            res.calls += 1
            st.last = ser[k - 1]
            st.time = ser[k - 1].time
            done += k
            istep += k
            if mdmod(istep, ctl.nckpt) == 0:
                ckpt(istep)
        engine.cancel_vcom()                                 # md.F:94-95
        engine.tnorm()
        res.warmup.append((istep, st.time))
    if istep > 0 and mdmod(istep, ctl.nckpt) != 0:
        ckpt(istep)

    # -- measurement (md.F:122-166) ---------------------------------------
    evave = ev2ave = pave = p2ave = 0.0
    istep = 0
    wrapped = False
    per_group = ctl.ntot * ctl.nind
    for ig in range(1, ctl.ngroup + 1):
        eva = ev2a = pa = p2a = 0.0
        gend = ig * per_group
        while istep < gend:
            if mdmod(istep, ctl.ncom) == 0:
                engine.cancel_vcom()
            if mdmod(istep, ctl.ntnorm) == 0:
                engine.tnorm()
            if ctl.strained or not wrapped:
                engine.strain(ctl.deps, xl0)
                wrapped = True
            # next step at which md.F does something on the host
            b = gend
            if ctl.strained:
                b = istep + 1
            for q in (ctl.ncom, ctl.ntnorm, ctl.nout, ctl.nckpt):
                if q > 0:
                    b = min(b, (istep // q + 1) * q)
            t0 = istep
            for k, m in plan(istep, b, ctl.nind, ctl.nptensor):
                ser = engine.run(k, m, series=True)
                res.calls += 1
                for j in range(k):
                    sc = ser[j]
                    i1 = t0 + j + 1
                    if measures(i1, ctl.nind, ctl.nptensor):
                        if mdmod(i1, ctl.nind) == 0:
                            eva += sc.ev
                            ev2a += sc.ev ** 2
                            pa += sc.px
                            p2a += sc.px ** 2
                            res.e_lines.append((i1, sc.time, sc.ev, sc.ek, sc.ek + sc.ev, sc.px))
                        if mdmod(i1, ctl.nptensor) == 0:
                            res.p_lines.append((i1, sc.time) + _pp6(sc))
                        res.meas.append((i1, sc.time, sc.ev, sc.ek, sc.px) + _pp6(sc))
                st.last = ser[k - 1]
                st.time = ser[k - 1].time
                t0 += k
            istep = b
            if mdmod(istep, ctl.nout) == 0 and on_save is not None:
                on_save(engine, istep, st.time, st.last)
            if mdmod(istep, ctl.nckpt) == 0:
                ckpt(istep)
        eva, ev2a, dev, evave, ev2ave = statt(eva, ev2a, ctl.ntot, evave, ev2ave)
        pa, p2a, dp, pave, p2ave = statt(pa, p2a, ctl.ntot, pave, p2ave)
        res.groups.append((ig, st.time, eva, dev, pa, dp))
    if ctl.ngroup > 0:
        res.evave, _, res.devave, _, _ = statt(evave, ev2ave, ctl.ngroup, 0.0, 0.0)
        res.pave, _, res.dpave, _, _ = statt(pave, p2ave, ctl.ngroup, 0.0, 0.0)
    if istep > 0 and mdmod(istep, ctl.nckpt) != 0:
        ckpt(istep)

    s = engine.accel(True)                                   # md.F:188-190
    ek = engine.ttot()
    xl = list(engine.params.xl)
    res.final = dict(xl=xl, stretch=[xl[k] / xl0[k] for k in range(3)],
                     rho=f_float(n) / (xl[0] * xl[1] * xl[2]),
                     ev=s.ev, ek=ek, e=s.ev + ek, px=s.px)
    return res


def format_e_line(tag, istep, time, vals):
    """md.F:10101 format(a1,1x,i7,1x,f14.2,6(2x,es16.9))."""
    return "%s %7d %14.2f" % (tag, istep, time) + "".join("  %16.9E" % v for v in vals)
