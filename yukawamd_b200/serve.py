"""Serving loop: continuous batching of MD runs on one GPU.

A request is one MD run: a box (configs.Workload), a number of
velocity-Verlet steps and a precision.  The server keeps one group per
(kind, precision) -- ion or nucleon boxes, mixed or FP64 -- and every group
is one device-resident batch of fixed capacity (engine.SlotBatch: slots,
particles and half-pair scratch reserved once, from an HBM budget split
between the groups).  Each group runs in its own host thread on its own CUDA
stream, independently of the others:

  * between chunks it admits waiting requests of its kind into free slots
    (yk_batch_admit copies the new run's initial state in, orders it and makes
    its initial force call, md.F:69, over its own work items only);
  * it advances every run it holds by one chunk of up to `chunk` steps, one
    CUDA graph; each run stops at exactly its own step count inside the
    graph (a per-box step budget on the device), so a chunk never has to be
    shortened for the run that ends first;
  * it retires the runs whose budget is spent (their final state is copied
    out, their slot freed).
Runs that stay are never moved, copied through the host or recomputed: one
force call per step (vel_verlet_2.f:58) and no other.

Admission is first come, first served with a bounded bypass: a request that
does not fit yet lets later, smaller requests of the same group in, until it
has waited `max_bypass_s`; then nothing passes it.

The energy of every run is taken at the end of every chunk (the chunk's last
step measures); 1 in `shadow_every` mixed runs can get an FP64 twin, and both
runs' drift is reported.

A run's arithmetic depends only on its own box: its slot order comes from a
sort of its own particles, its work items write only its own scratch, and
its chunks start when it is admitted, so its result is the same bits alone or
in a mix (tests/test_serve.py).

Reported: p50 / p99 completion latency (arrival to completion, wall clock),
aggregate pair interactions per second, per-run results, and per group the
admissions and the wall time they took.
"""
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from . import abi
from ._lib import EngineError
from .engine import SlotBatch

PB = 128
# device bytes per particle of a group's reserved state and slot arrays
PARTICLE_BYTES = 300


def unit_bytes(precision=abi.YK_PREC_FP64):
    """Device bytes per half-pair unit of reserved scratch: the source-side
    row (128 x 3 values: doubles in the FP64 form, floats in the mixed form)
    plus the target-side rows (doubles) and job entries at the default
    segment length (a quarter of a double row at most) and slack."""
    sj = 3 * PB * (4 if precision == abi.YK_PREC_MIXED else 8)
    return sj + 3 * PB * 8 // 4 + 64


def pair_units(n):
    t = (int(n) + PB - 1) // PB
    return t * (t + 1) // 2


def footprint_bytes(n, precision=abi.YK_PREC_FP64):
    """Device bytes a run of n particles takes inside a group: its state
    and slot arrays plus its half-pair scratch."""
    t = (int(n) + PB - 1) // PB
    return PARTICLE_BYTES * (n + 3) + 84 * PB * t + unit_bytes(precision) * pair_units(n)


@dataclass
class Request:
    rid: int
    workload: object
    steps: int
    precision: int = abi.YK_PREC_MIXED
    arrival: float = 0.0
    shadow_of: int = -1              # rid of the run this FP64 twin shadows
    # filled by the server
    admitted: float = None
    done: float = None
    steps_done: int = 0
    energies: list = field(default_factory=list)   # (step, E per particle)
    final_x: np.ndarray = None
    final_v: np.ndarray = None
    slot: int = -1
    group: tuple = None

    @property
    def kind(self):
        return "nucleon" if self.workload.params["sim_type"] == abi.YK_SIM_NUCLEON else "ion"

    @property
    def key(self):
        return (self.kind, self.precision)

    @property
    def n(self):
        return self.workload.n

    @property
    def pairs(self):
        return self.steps * self.n * (self.n - 1) // 2

    @property
    def latency(self):
        return None if self.done is None else self.done - self.arrival


def pick(waiting, fits, now, max_bypass_s):
    """Admission order of one group: scan `waiting` (arrival order) and take
    every request for which fits(r) is true.  A request that does not fit is
    passed over, but once one that does not fit has waited max_bypass_s
    (now - arrival), no later request is taken.  Returns the taken ones.
    fits() may keep state (it is called in order and may account for the
    requests already taken)."""
    out = []
    for r in waiting:
        if fits(r):
            out.append(r)
        elif now - r.arrival >= max_bypass_s:
            break
    return out


def admit(waiting, active_bytes, budget):
    """Footprint admission against one budget: the requests of `waiting`
    (arrival order) that fit, passing over those that do not (pick with no
    bypass limit).  Returns (admitted requests, new active bytes)."""
    used = [active_bytes]

    def fits(r):
        need = footprint_bytes(r.n, r.precision)
        if used[0] + need > budget:
            return False
        used[0] += need
        return True
    got = pick(waiting, fits, 0.0, float("inf"))
    return got, used[0]


# Share of the HBM budget that each group reserves: mixed runs carry the
# load, FP64 groups hold the shadow twins.
GROUP_SHARE = {("ion", abi.YK_PREC_MIXED): 0.45, ("nucleon", abi.YK_PREC_MIXED): 0.30,
               ("ion", abi.YK_PREC_FP64): 0.15, ("nucleon", abi.YK_PREC_FP64): 0.10}


class Group:
    """One device-resident batch and the runs it holds."""

    def __init__(self, key, proto, budget_bytes, device, nslots, chunk, autotune):
        self.key = key
        self.chunk = chunk
        self.max_particles = max(PB, int(0.05 * budget_bytes) // PARTICLE_BYTES)
        part_bytes = PARTICLE_BYTES * self.max_particles
        self.max_units = max(1, (budget_bytes - part_bytes) // unit_bytes(key[1]))
        self.batch = SlotBatch(proto, nslots, self.max_particles, self.max_units, device=device)
        if autotune:
            from . import tune
            tune.apply_batch(self.batch, device)
        self.batch.set_tuning(graph_steps=chunk)          # one CUDA graph per chunk
        self.members = {}                                  # slot -> Request
        self.admissions = 0
        self.admit_s = 0.0
        self.chunks = 0
        self.pairs = 0

    def fits(self, r):
        return r.n <= self.max_particles and pair_units(r.n) <= self.max_units

    def try_admit(self, r, t0):
        w = r.workload
        p = w.yk_params(precision=r.precision, mix_mode=abi.YK_MIX_FIXED)
        t = time.perf_counter()
        try:
            slot, _s = self.batch.admit(p, w.x, w.v, w.zii, w.aii, r.steps)
        except EngineError as e:
            if e.code == abi.YK_ERR_NOMEM:
                return False
            raise
        finally:
            self.admit_s += time.perf_counter() - t
        r.slot = slot
        r.group = self.key
        r.admitted = time.perf_counter() - t0
        self.members[slot] = r
        self.admissions += 1
        return True

    def step(self, t0):
        """One chunk; returns the runs that finished in it."""
        k = self.chunk
        ser, _ms = self.batch.run(k, k, series=True)
        left = self.batch.steps_left()
        nsl = self.batch.nrep
        done = []
        for slot, r in list(self.members.items()):
            took = min(k, r.steps - r.steps_done)
            self.pairs += took * r.n * (r.n - 1) // 2
            r.steps_done += took
            if took == k:
                s = ser[(k - 1) * nsl + slot]
                r.energies.append((r.steps_done, s.ev + s.ek))
            if left[slot] == 0:
                x, v, _vold, _a = self.batch.retire(slot)
                r.final_x, r.final_v = x, v
                r.done = time.perf_counter() - t0
                del self.members[slot]
                done.append(r)
        self.chunks += 1
        return done

    def close(self):
        self.batch.close()


class Server:
    def __init__(self, device=0, hbm_budget=None, chunk=50, shadow_every=16, autotune=False, nslots=256,
                 max_bypass_s=2.0):
        self.device = device
        self.chunk = chunk
        self.shadow_every = shadow_every
        self.autotune = autotune          # apply cached batch tunings (tune.apply_batch)
        self.nslots = nslots
        self.max_bypass_s = max_bypass_s
        if hbm_budget is None:
            import torch
            free, _total = torch.cuda.mem_get_info(device)
            hbm_budget = int(0.6 * free)
        self.budget = hbm_budget
        self.groups = {}
        self.finished = []

    def _group(self, key, r, share):
        proto = r.workload.yk_params(precision=r.precision)
        g = Group(key, proto, int(share * self.budget), self.device, self.nslots, self.chunk, self.autotune)
        self.groups[key] = g
        return g

    def run(self, requests, time_scale=1.0):
        """Serve `requests` (their .arrival in seconds after the start, scaled
        by time_scale).  Returns a report dict."""
        pending = sorted(requests, key=lambda r: r.arrival)
        keys = sorted(set(r.key for r in pending))
        total = sum(GROUP_SHARE.get(k, 0.1) for k in keys)
        for key in keys:
            self._group(key, next(r for r in pending if r.key == key), GROUP_SHARE.get(key, 0.1) / total)
        lock = threading.Condition()
        waiting = {key: [] for key in keys}
        remaining = {key: sum(1 for r in pending if r.key == key) for key in keys}
        state = {"error": None}
        t0 = time.perf_counter()

        def feeder():
            for r in pending:
                delay = r.arrival * time_scale - (time.perf_counter() - t0)
                if delay > 0:
                    time.sleep(delay)
                with lock:
                    waiting[r.key].append(r)
                    lock.notify_all()

        def worker(key):
            g = self.groups[key]
            try:
                while True:
                    with lock:
                        while not waiting[key] and not g.members and remaining[key] > 0 and not state["error"]:
                            lock.wait(timeout=0.05)
                        if state["error"] or remaining[key] == 0:
                            return
                        queue = list(waiting[key])
                    now = time.perf_counter() - t0
                    taken = pick(queue, lambda r: g.fits(r) and g.try_admit(r, t0), now, self.max_bypass_s)
                    if taken:
                        with lock:
                            for r in taken:
                                waiting[key].remove(r)
                    if not g.members:
                        if queue and not taken and not any(g.fits(r) for r in queue):
                            raise RuntimeError("a request does not fit its group's capacity: n = %d"
                                               % max(r.n for r in queue))
                        time.sleep(0.001)
                        continue
                    done = g.step(t0)
                    if done:
                        with lock:
                            self.finished.extend(done)
                            remaining[key] -= len(done)
                            lock.notify_all()
            except BaseException as e:       # surface worker failures in run()
                with lock:
                    state["error"] = e
                    lock.notify_all()

        threads = [threading.Thread(target=feeder, daemon=True)]
        threads += [threading.Thread(target=worker, args=(key,), daemon=True) for key in keys]
        for th in threads:
            th.start()
        for th in threads[1:]:
            th.join()
        wall = time.perf_counter() - t0
        threads[0].join(timeout=1.0)
        pairs = sum(g.pairs for g in self.groups.values())
        rep = self.report(wall, pairs)
        for g in self.groups.values():
            g.close()
        self.groups = {}
        if state["error"] is not None:
            raise state["error"]
        return rep

    def report(self, wall, pairs_done):
        lat = np.array([r.latency for r in self.finished if r.shadow_of < 0])
        out = {"runs": len(lat), "wall_s": wall, "pairs": pairs_done,
               "pairs_per_s": pairs_done / wall if wall > 0 else 0.0,
               "latency_p50_s": float(np.percentile(lat, 50)) if len(lat) else None,
               "latency_p99_s": float(np.percentile(lat, 99)) if len(lat) else None,
               "latency_max_s": float(lat.max()) if len(lat) else None,
               "groups": {"%s/%s" % (k[0], "mixed" if k[1] == abi.YK_PREC_MIXED else "fp64"):
                          {"admissions": g.admissions, "admit_wall_s": g.admit_s, "chunks": g.chunks,
                           "slots": g.batch.nrep, "max_particles": g.max_particles,
                           "max_pair_units": g.max_units}
                          for k, g in self.groups.items()}}
        shadows = []
        by_id = {r.rid: r for r in self.finished}
        for r in self.finished:
            if r.shadow_of >= 0 and r.shadow_of in by_id:
                m = by_id[r.shadow_of]
                shadows.append({"rid": m.rid, "n": m.n, "steps": m.steps,
                                "drift_mixed": drift(m.energies), "drift_fp64": drift(r.energies)})
        out["fp64_shadows"] = shadows
        return out


def drift(energies):
    """max |E(step) - E(first)| / |E(first)| over the recorded chunk ends."""
    if len(energies) < 2:
        return 0.0
    e = np.array([t[1] for t in energies])
    return float(np.max(np.abs(e - e[0])) / abs(e[0]))


def make_requests(stream, shadow_every=16):
    """Requests from configs.request_stream output [(arrival, workload)]:
    mixed precision, with an FP64 twin for every shadow_every-th run."""
    reqs = []
    rid = 0
    for k, (t, w) in enumerate(stream):
        reqs.append(Request(rid, w, w.steps, abi.YK_PREC_MIXED, t))
        if shadow_every and k % shadow_every == 0:
            reqs.append(Request(rid + 1, w, w.steps, abi.YK_PREC_FP64, t, shadow_of=rid))
            rid += 1
        rid += 1
    return reqs
