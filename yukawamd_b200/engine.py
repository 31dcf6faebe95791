"""Host-side mirror of the reference's force-call and integrator interface.

The Fortran code calls two argument-less routines that work on module
globals (md_globals.f:153-172):

    call accel(do_measurements)     ! int_control.f:52-81
    call newton(do_measurements)    ! vel_verlet_2.f:18-120

Engine keeps the same shape: the particle arrays live on the device, the
scalar results (ev, vir, px, ek, pp, time) come back as attributes after each
call, and errors raise EngineError carrying the C-ABI status, the way the
Fortran shim maps them to md_exit.
"""
import ctypes as C

import numpy as np

from . import abi
from ._lib import check, check_batch, lib

_dp = C.POINTER(C.c_double)


def _ptr(a):
    if a is None:
        return None
    if a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"]:
        raise TypeError("arrays must be C-contiguous float64")
    return a.ctypes.data_as(_dp)


def _f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64).reshape(-1)


class Engine:
    """One simulation box on one GPU.

    params: abi.YkParams (or a configs.Workload, whose arrays are then used
    when x is None).  x, v: double[3n] in the Fortran layout x(3,0:n-1).
    """

    def __init__(self, params, x=None, v=None, zii=None, aii=None, **overrides):
        if not isinstance(params, abi.YkParams):
            w = params
            params = w.yk_params(**overrides)
            x = w.x if x is None else x
            v = w.v if v is None else v
            zii = w.zii if zii is None else zii
            aii = w.aii if aii is None else aii
        else:
            for k, val in overrides.items():
                setattr(params, k, val)
        self.params = params
        x, v, zii, aii = _f64(x), _f64(v), _f64(zii), _f64(aii)
        if x is None:
            raise ValueError("positions are required")
        self.n = len(x) // 3
        self._lib = lib()
        self._ctx = C.c_void_p()
        check(self._lib.yk_create(C.byref(params), self.n, _ptr(x), _ptr(v), _ptr(zii),
                                  _ptr(aii), C.byref(self._ctx)))
        self.scalars = abi.YkScalars()
        self.a = np.zeros(3 * (self.n + 3))

    # -- the reference's two entry points ---------------------------------
    def accel(self, do_measurements=True, fetch_a=True):
        """accel(do_measurements): forces from the device-resident positions.
        Fills self.a (double[3(n+3)], the reference layout) when fetch_a."""
        check(self._lib.yk_accel(self._ctx, int(bool(do_measurements)),
                                 _ptr(self.a) if fetch_a else None,
                                 C.byref(self.scalars)), self._ctx)
        return self.scalars

    def newton(self, do_measurements=False):
        """newton(do_measurements): one integrator step on the device."""
        check(self._lib.yk_newton(self._ctx, int(bool(do_measurements)),
                                  C.byref(self.scalars)), self._ctx)
        return self.scalars

    # -- device-resident stepping ---------------------------------------
    def run(self, nsteps, meas_every=0, series=True):
        """nsteps steps launched as CUDA graphs; returns the per-step scalars
        (a ctypes array of YkScalars) when series, else None."""
        buf = (abi.YkScalars * nsteps)() if series and nsteps > 0 else None
        check(self._lib.yk_run(self._ctx, int(nsteps), int(meas_every),
                               buf if buf is not None else None), self._ctx)
        if buf is not None and nsteps > 0:
            self.scalars = buf[nsteps - 1]
        return buf

    # -- sync points ------------------------------------------------------
    def get_state(self):
        n3 = 3 * self.n
        x, v, vold, a = (np.empty(n3) for _ in range(4))
        check(self._lib.yk_get_state(self._ctx, _ptr(x), _ptr(v), _ptr(vold), _ptr(a)),
              self._ctx)
        return x, v, vold, a

    def get_into(self, x=None, v=None, vold=None, a=None):
        check(self._lib.yk_get_state(self._ctx, _ptr(x), _ptr(v), _ptr(vold), _ptr(a)),
              self._ctx)

    def set_state(self, x=None, v=None, vold=None, a=None):
        x, v, vold, a = _f64(x), _f64(v), _f64(vold), _f64(a)
        if a is not None and len(a) == 3 * (self.n + 3):
            a = np.ascontiguousarray(a[:3 * self.n])
        check(self._lib.yk_set_state(self._ctx, _ptr(x), _ptr(v), _ptr(vold), _ptr(a)),
              self._ctx)

    def set_box(self, xl):
        arr = (C.c_double * 3)(*[float(t) for t in xl])
        check(self._lib.yk_set_box(self._ctx, C.cast(arr, _dp)), self._ctx)
        for k in range(3):
            self.params.xl[k] = float(xl[k])

    # -- asynchronous snapshots (checkpoint / save_config) ------------------
    def snapshot_begin(self, x=None, v=None, a=None):
        """Start copying x, v, a (host float64 arrays of 3n, written in place)
        from the device; returns at once.  The arrays hold the snapshot after
        snapshot_wait()."""
        for t in (x, v, a):
            if t is not None and t.size != 3 * self.n:
                raise ValueError("snapshot arrays hold 3*n doubles")
        check(self._lib.yk_snapshot_begin(self._ctx, _ptr(x), _ptr(v), _ptr(a)), self._ctx)
        self._snap_refs = (x, v, a)        # keep the targets alive while the copy runs

    def snapshot_wait(self):
        check(self._lib.yk_snapshot_wait(self._ctx), self._ctx)
        self._snap_refs = None

    # -- gen_utils.f / strain.f on the device ------------------------------
    def ttot(self):
        out = C.c_double()
        check(self._lib.yk_ttot(self._ctx, C.byref(out)), self._ctx)
        return out.value

    def vtot(self):
        """(ev, px) of the current positions; the accelerations are not changed."""
        ev, px = C.c_double(), C.c_double()
        check(self._lib.yk_vtot(self._ctx, C.byref(ev), C.byref(px)), self._ctx)
        return ev.value, px.value

    def gofr_counts(self, nbin, counts=None):
        """Add the pair-distance histogram of g(r) (g.f:55-66) of the current
        positions to counts (float64[nbin], new zeros if None); returns it."""
        counts = np.zeros(int(nbin)) if counts is None else counts
        if counts.dtype != np.float64 or counts.size != int(nbin) or not counts.flags["C_CONTIGUOUS"]:
            raise ValueError("counts must be a C-contiguous float64 array of nbin values")
        check(self._lib.yk_gofr_counts(self._ctx, int(nbin), _ptr(counts)), self._ctx)
        return counts

    def tnorm(self):
        check(self._lib.yk_tnorm(self._ctx), self._ctx)

    def cancel_vcom(self):
        check(self._lib.yk_cancel_vcom(self._ctx), self._ctx)

    def strain(self, deps, xl0):
        d = (C.c_double * 3)(*[float(t) for t in deps])
        g = (C.c_double * 3)(*[float(t) for t in xl0])
        out = (C.c_double * 3)()
        check(self._lib.yk_strain(self._ctx, C.cast(d, _dp), C.cast(g, _dp), C.cast(out, _dp)), self._ctx)
        for k in range(3):
            self.params.xl[k] = out[k]
        return list(out)

    # -- engine tunables (force kernel, job size, sort cadence, graph length) -
    def tuning(self):
        t = abi.YkTuning()
        check(self._lib.yk_get_tuning(self._ctx, C.byref(t)), self._ctx)
        return t

    def set_tuning(self, force_kernel=None, pair_seg=None, sort_every=None, graph_steps=None,
                   source_split=None, targets_per_thread=None):
        t = self.tuning()
        for name, val in (("force_kernel", force_kernel), ("pair_seg", pair_seg),
                          ("sort_every", sort_every), ("graph_steps", graph_steps),
                          ("source_split", source_split), ("targets_per_thread", targets_per_thread)):
            if val is not None:
                setattr(t, name, int(val))
        check(self._lib.yk_set_tuning(self._ctx, C.byref(t)), self._ctx)
        return self.tuning()

    # -- timers (the reference's perf.f newton / accel timers) --------------
    def perf_enable(self, enable=True, flush_bytes=0):
        check(self._lib.yk_perf_enable(self._ctx, int(bool(enable)), int(flush_bytes)),
              self._ctx)

    def perf_read(self):
        out = abi.YkPerf()
        check(self._lib.yk_perf_read(self._ctx, C.byref(out)), self._ctx)
        return out

    @property
    def time(self):
        return self.scalars.time

    def close(self):
        if self._ctx:
            self._lib.yk_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many independent boxes advanced together (one persistent force kernel
    over all boxes' work items, CUDA graphs of K steps).  boxes: a list of
    configs.Workload, or of (YkParams, x, v, zii, aii) tuples."""

    def __init__(self, boxes, device=0, **overrides):
        params, xs, vs, zs, ms = [], [], [], [], []
        for b in boxes:
            if isinstance(b, tuple):
                p, x, v, z, m = b
            else:
                p = b.yk_params(**overrides)
                x, v, z, m = b.x, b.v, b.zii, b.aii
            params.append(p)
            xs.append(_f64(x))
            vs.append(_f64(v))
            zs.append(_f64(z))
            ms.append(_f64(m))
        self.nrep = len(params)
        self.n = [len(x) // 3 for x in xs]
        self._keep = (xs, vs, zs, ms)
        P = (abi.YkParams * self.nrep)(*params)
        self.params = P
        N = (C.c_int * self.nrep)(*self.n)

        def ptrs(arrs):
            return (_dp * self.nrep)(*[_ptr(a) if a is not None else None for a in arrs])
        self._lib = lib()
        self._b = C.c_void_p()
        check_batch(self._lib.yk_batch_create(self.nrep, P, N, ptrs(xs), ptrs(vs), ptrs(zs), ptrs(ms),
                                              int(device), C.byref(self._b)))
        self._keep = None

    def tuning(self):
        t = abi.YkTuning()
        check_batch(self._lib.yk_batch_get_tuning(self._b, C.byref(t)), self._b)
        return t

    def set_tuning(self, pair_seg=None, graph_steps=None, sort_every=None):
        t = self.tuning()
        if pair_seg is not None:
            t.pair_seg = int(pair_seg)
        if graph_steps is not None:
            t.graph_steps = int(graph_steps)
        if sort_every is not None:
            t.sort_every = int(sort_every)
        check_batch(self._lib.yk_batch_set_tuning(self._b, C.byref(t)), self._b)
        return self.tuning()

    def accel(self, do_measurements=True):
        out = (abi.YkScalars * self.nrep)()
        check_batch(self._lib.yk_batch_accel(self._b, int(bool(do_measurements)), out), self._b)
        return out

    def run(self, nsteps, meas_every=0, series=True):
        """Returns (series or None, milliseconds of device time); series is a
        ctypes array indexed [step * nrep + box]."""
        buf = (abi.YkScalars * (nsteps * self.nrep))() if series and nsteps > 0 else None
        ms = C.c_double()
        check_batch(self._lib.yk_batch_run(self._b, int(nsteps), int(meas_every), buf, C.byref(ms)),
                    self._b)
        return buf, ms.value

    def get_state(self, rep):
        n = self.n[rep]
        x, v, vold = (np.empty(3 * n) for _ in range(3))
        a = np.empty(3 * (n + 3))
        check_batch(self._lib.yk_batch_get_state(self._b, int(rep), _ptr(x), _ptr(v), _ptr(vold),
                                                 _ptr(a)), self._b)
        return x, v, vold, a

    def set_state(self, rep, x=None, v=None, vold=None, a=None):
        x, v, vold, a = _f64(x), _f64(v), _f64(vold), _f64(a)
        check_batch(self._lib.yk_batch_set_state(self._b, int(rep), _ptr(x), _ptr(v), _ptr(vold),
                                                 _ptr(a)), self._b)

    def close(self):
        if self._b:
            self._lib.yk_batch_destroy(self._b)
            self._b = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SlotBatch(Batch):
    """A batch of fixed capacity that runs enter and leave one at a time
    (yk_batch_create_slots / yk_batch_admit / yk_batch_retire): the serving
    loop's device-resident group.  proto: YkParams of the kind (ion or
    nucleon) and precision of every box it will hold.  Slots are indexed
    0 .. nslots-1; run()'s series is indexed [step * nslots + slot]."""

    def __init__(self, proto, nslots, max_particles, max_pair_units, device=0):
        self._lib = lib()
        self._b = C.c_void_p()
        self.nrep = int(nslots)
        self.n = [0] * self.nrep
        check_batch(self._lib.yk_batch_create_slots(C.byref(proto), self.nrep, int(max_particles),
                                                    int(max_pair_units), int(device), C.byref(self._b)))

    @staticmethod
    def pair_units(n):
        t = (int(n) + 127) // 128
        return t * (t + 1) // 2

    def admit(self, params, x, v, zii, aii, steps):
        """Admit one box with a budget of `steps` steps; returns (slot, its
        scalars after the initial measuring force call).  Raises EngineError
        with code YK_ERR_NOMEM when it does not fit."""
        x, v, zii, aii = _f64(x), _f64(v), _f64(zii), _f64(aii)
        n = len(x) // 3
        slot = C.c_int(-1)
        out = abi.YkScalars()
        check_batch(self._lib.yk_batch_admit(self._b, C.byref(params), n, _ptr(x), _ptr(v), _ptr(zii), _ptr(aii),
                                             int(steps), C.byref(slot), C.byref(out)), self._b)
        self.n[slot.value] = n
        return slot.value, out

    def retire(self, slot):
        """The box's final (x, v, vold, a); its slot is free afterwards."""
        n = self.n[slot]
        x, v, vold = (np.empty(3 * n) for _ in range(3))
        a = np.empty(3 * (n + 3))
        check_batch(self._lib.yk_batch_retire(self._b, int(slot), _ptr(x), _ptr(v), _ptr(vold), _ptr(a)),
                    self._b)
        self.n[slot] = 0
        return x, v, vold, a

    def steps_left(self):
        """Remaining step budget per slot (-1 for an empty slot)."""
        out = (C.c_int * self.nrep)()
        check_batch(self._lib.yk_batch_steps_left(self._b, out), self._b)
        return np.array(out[:], dtype=np.int64)


def kernel_launch_count():
    return int(lib().yk_kernel_launch_count())


def peak_probe(device=0, kind=0):
    """Measured FMA throughput of the GPU in TFLOP/s (kind 0 FP64, 1 FP32)."""
    out = C.c_double()
    check(lib().yk_peak_probe(int(device), int(kind), C.byref(out)))
    return out.value


def pair_jobs(m, cap, ctas, targets_per_thread=1):
    """The half-pair kernel's job table for m tiles (yk_pair_jobs, or
    yk_pair_jobs2 for two targets per thread): an int array of shape (jobs, 4)
    with rows (R, C0, C1, slot) in dispatch order, and the Si slot count of
    every row.  Host arithmetic only."""
    fn = lib().yk_pair_jobs2 if targets_per_thread == 2 else lib().yk_pair_jobs
    k = fn(int(m), int(cap), int(ctas), None, 0, None)
    if k < 0:
        raise ValueError("yk_pair_jobs: bad arguments (m=%r, cap=%r, ctas=%r)" % (m, cap, ctas))
    jobs = np.zeros((k, 4), dtype=np.int32)
    slots = np.zeros(int(m), dtype=np.int32)
    got = fn(int(m), int(cap), int(ctas), jobs.ctypes.data_as(C.POINTER(C.c_int)), k,
             slots.ctypes.data_as(C.POINTER(C.c_int)))
    assert got == k
    return jobs, slots


def accel_noalloc(params, n, x_dev, zii_dev, aii_dev, do_measurements, a_dev, stream=None):
    """Force call on caller-owned device arrays (raw device addresses as ints)
    that allocates no device memory; see yk_accel_noalloc in
    include/yukawa_engine.h for who needs it and its limits (n <= 4096, calls
    must not overlap on the GPU).  Returns the scalars."""
    out = abi.YkScalars()
    check(lib().yk_accel_noalloc(C.byref(params), int(n), x_dev, zii_dev, aii_dev,
                                 int(bool(do_measurements)), a_dev, C.byref(out), stream))
    return out


def version():
    return lib().yk_version().decode()


def host_register(arr):
    check(lib().yk_host_register(arr.ctypes.data_as(C.c_void_p), arr.nbytes))


def host_unregister(arr):
    check(lib().yk_host_unregister(arr.ctypes.data_as(C.c_void_p)))
