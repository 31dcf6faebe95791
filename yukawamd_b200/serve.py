"""Serving loop: continuous batching of MD runs on one GPU.

A request is one MD run: a box (configs.Workload), a number of
velocity-Verlet steps and a precision.  The server

  * admits waiting requests (first come, first served) while the estimated
    device footprint of all admitted runs fits an HBM budget;
  * keeps every admitted run's state resident on the device, grouped into
    batch engines (yukawamd_b200.engine.Batch) by kind (ion / nucleon) and
    precision, and advances all groups concurrently (one host thread and one
    CUDA stream per group, so their kernels overlap on the GPU);
  * advances in chunks of at most `chunk` steps; between chunks, finished runs
    leave and newly admitted runs join (the groups are rebuilt; continuing
    runs carry their exact x, v, vold and a across the rebuild);
  * measures the energy at the end of every chunk of every run;
  * optionally runs an FP64 twin of 1 in `shadow_every` mixed-precision runs
    and reports both runs' energy drift.

Each run's arithmetic depends only on its own box, so its result is the same
alone or in the mix up to the summation order chosen by the Morton ordering
(which is refreshed at group rebuilds); tests/test_serve.py states and
checks the tolerance.

Reported: p50 / p99 completion latency (arrival to completion, wall clock),
aggregate pair interactions per second, and per-run results.
"""
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from . import abi
from .engine import Batch

PB = 128


def footprint_bytes(n, seg=8):
    """Device bytes a box of n particles holds inside a batch: state and
    slot arrays (~260 B per particle; 84 B per slot: FP64 positions and the
    FP32 shadow) plus the half-pair scratch."""
    t = (n + PB - 1) // PB
    nseg = (t + seg - 1) // seg
    scratch = 8 * 3 * PB * (t * (t + 1) // 2 + t * nseg)
    return 260 * n + 84 * PB * t + scratch + 4096


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
    state: tuple = None              # (x, v, vold, a) between chunks

    @property
    def kind(self):
        return "nucleon" if self.workload.params["sim_type"] == abi.YK_SIM_NUCLEON else "ion"

    @property
    def n(self):
        return self.workload.n

    @property
    def pairs(self):
        return self.steps * self.n * (self.n - 1) // 2

    @property
    def latency(self):
        return None if self.done is None else self.done - self.arrival


def admit(waiting, active_bytes, budget, seg=8):
    """FIFO admission by footprint: the longest prefix of `waiting` that fits.
    Returns (admitted requests, new active bytes)."""
    out = []
    for r in waiting:
        need = footprint_bytes(r.n, seg)
        if active_bytes + need > budget:
            break
        out.append(r)
        active_bytes += need
    return out, active_bytes


class Server:
    def __init__(self, device=0, hbm_budget=None, chunk=50, shadow_every=16, autotune=False):
        self.device = device
        self.chunk = chunk
        self.shadow_every = shadow_every
        self.autotune = autotune          # apply cached batch tunings (tune.apply_batch)
        if hbm_budget is None:
            import torch
            free, _total = torch.cuda.mem_get_info(device)
            hbm_budget = int(0.6 * free)
        self.budget = hbm_budget
        self.groups = {}          # (kind, precision) -> (Batch, [Request])
        self.finished = []
        self.rebuilds = 0         # group rebuilds and the wall time spent in them
        self.rebuild_s = 0.0

    # -- group management ----------------------------------------------
    def _rebuild(self, key, runs):
        old = self.groups.pop(key, None)
        if old is not None:
            batch, members = old
            for i, r in enumerate(members):
                if r.done is None:
                    r.state = batch.get_state(i)
            batch.close()
        if not runs:
            return
        boxes = []
        fresh = []
        for r in runs:
            w = r.workload
            p = w.yk_params(precision=r.precision, mix_mode=abi.YK_MIX_FIXED)
            p.time = w.params.get("time", 0.0) + r.steps_done * p.dt
            if r.state is None:
                boxes.append((p, w.x, w.v, w.zii, w.aii))
                fresh.append(True)
            else:
                x, v, vold, a = r.state
                boxes.append((p, x, v, w.zii, w.aii))
                fresh.append(False)
        batch = Batch(boxes, device=self.device)
        if self.autotune:
            from . import tune
            tune.apply_batch(batch, self.device)
        batch.set_tuning(graph_steps=self.chunk)      # one CUDA graph per chunk
        batch.accel(True)                            # md.F:69 for the new runs
        for i, r in enumerate(runs):
            if not fresh[i]:
                x, v, vold, a = r.state
                batch.set_state(i, vold=vold, a=a)   # continuing runs keep their a
        self.groups[key] = (batch, list(runs))

    def _advance(self, key, k):
        batch, members = self.groups[key]
        ser, _ms = batch.run(k, k, series=True)
        last = (k - 1) * batch.nrep
        for i, r in enumerate(members):
            s = ser[last + i]
            r.steps_done += k
            r.energies.append((r.steps_done, s.ev + s.ek))

    # -- the loop ----------------------------------------------------------
    def run(self, requests, time_scale=1.0):
        """Serve `requests` (their .arrival in seconds after the start, scaled
        by time_scale).  Returns a report dict."""
        pending = sorted(requests, key=lambda r: r.arrival)
        waiting, active = [], []
        active_bytes = 0
        t0 = time.perf_counter()
        pairs_done = 0
        while pending or waiting or active:
            now = time.perf_counter() - t0
            while pending and pending[0].arrival * time_scale <= now:
                waiting.append(pending.pop(0))
            if not active and not waiting:
                time.sleep(max(0.0, pending[0].arrival * time_scale - now))
                continue
            admitted, active_bytes = admit(waiting, active_bytes, self.budget)
            changed = bool(admitted)
            for r in admitted:
                waiting.remove(r)
                r.admitted = time.perf_counter() - t0
                active.append(r)
            if not active:
                # the head of the queue alone exceeds the budget: admit it anyway
                r = waiting.pop(0)
                r.admitted = time.perf_counter() - t0
                active.append(r)
                active_bytes += footprint_bytes(r.n)
                changed = True
            if changed:
                self._sync_groups(active)
            # one chunk: every group advances min(chunk, shortest remaining) steps
            steps = {key: min(self.chunk, min(r.steps - r.steps_done for r in members))
                     for key, (_b, members) in self.groups.items()}
            threads = [threading.Thread(target=self._advance, args=(key, k)) for key, k in steps.items()]
            for th in threads:
                th.start()
            for th in threads:
                th.join()
            for key, k in steps.items():
                pairs_done += sum(r.n * (r.n - 1) // 2 for r in self.groups[key][1]) * k
            done_now = [r for r in active if r.steps_done >= r.steps]
            if done_now:
                t_done = time.perf_counter() - t0
                for r in done_now:
                    batch, members = self.groups[(r.kind, r.precision)]
                    x, v, _vold, _a = batch.get_state(members.index(r))
                    r.final_x, r.final_v = x, v
                    r.done = t_done
                    r.state = None
                    active.remove(r)
                    active_bytes -= footprint_bytes(r.n)
                    self.finished.append(r)
                self._sync_groups(active)
        wall = time.perf_counter() - t0
        for key in list(self.groups):
            self._rebuild(key, [])
        return self.report(wall, pairs_done)

    def _sync_groups(self, active):
        """Rebuild exactly the groups whose membership changed."""
        t = time.perf_counter()
        keys = set((r.kind, r.precision) for r in active) | set(self.groups)
        for key in keys:
            want = [r for r in active if (r.kind, r.precision) == key]
            have = self.groups[key][1] if key in self.groups else []
            if [r.rid for r in want] != [r.rid for r in have]:
                self._rebuild(key, want)
                self.rebuilds += 1
        self.rebuild_s += time.perf_counter() - t

    def report(self, wall, pairs_done):
        lat = np.array([r.latency for r in self.finished if r.shadow_of < 0])
        out = {"runs": len(lat), "wall_s": wall, "pairs": pairs_done,
               "pairs_per_s": pairs_done / wall if wall > 0 else 0.0,
               "latency_p50_s": float(np.percentile(lat, 50)) if len(lat) else None,
               "latency_p99_s": float(np.percentile(lat, 99)) if len(lat) else None,
               "latency_max_s": float(lat.max()) if len(lat) else None,
               "group_rebuilds": self.rebuilds, "rebuild_wall_s": self.rebuild_s}
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
