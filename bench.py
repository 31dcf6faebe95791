#!/usr/bin/env python
"""Benchmark: pair-interactions/s of the velocity-Verlet step on one B200.

Workload (default): the ion mixture of MD 6.2.0's int_ion_mix.f at
N = 55,296 (Z = {6,8,26} with number fractions {0.2,0.7,0.1}, A = 2Z,
n = 7.18e-5 fm^-3, kappa = 0.5, effective Gamma = 150), all FP64.  One step
is one newton(do_measurements) of vel_verlet_2.f: drift, force call over all
N(N-1)/2 = 1,528,811,160 pairs, kick; it measures every --meas-every steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun (N > 1) every rank runs its own replica box on its own GPU
(replicas only: the path has no exchange step), the timed region is bracketed
by barriers and the time is the max over ranks.  Rank 0 prints one JSON line.

--impl reference times the reference's CPU algorithm, i.e. the OpenMP C
restatement in oracle/ (the Fortran cannot be compiled on these machines), on
all host cores, each step one whole force call over the same full-size box
(or, on hosts too slow for that, a block of target rows centred on the middle
row, which has the whole call's mean row length).
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

# The reference's mixture loops use schedule(runtime) (int_ion_mix.f:159,223);
# the CPU arms state the schedule they ran with and default it to static.
os.environ.setdefault("OMP_SCHEDULE", "static")

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

HEADLINE_METRIC = "pair-interactions/s mixed vs FP64 at <=1e-5 energy drift; served p99 latency"
UNIT = "pair-interactions/s"
# Algorithmic FP64 flops per unique pair (counted from the reference source,
# int_ion_pure.f:186-200 / :145-168, +2 for the mixture's Z weights).
FLOPS_PER_PAIR = {("mix", False): 30, ("mix", True): 47, ("ocp", False): 28, ("ocp", True): 45,
                  ("nucleon", False): 33, ("nucleon", True): 50}
L2_FLUSH_BYTES = 256 << 20


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["mix", "ocp", "nucleon"], default="mix")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--meas-every", type=int, default=10)
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--n", type=int, default=0,
                    help="override the particle count (same density; for profiling runs)")
    ap.add_argument("--no-companion", action="store_true",
                    help="skip the mixed-precision companion measurement")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the nucleon and replica-ensemble side measurements")
    ap.add_argument("--drift", type=int, default=0,
                    help="instead of the benchmark: run this many steps in FP64 and in mixed "
                         "precision and report the total-energy drift")
    ap.add_argument("--kernel", choices=["auto", "rows", "pairs", "near"], default="auto",
                    help="force kernel (default: the engine's automatic choice)")
    ap.add_argument("--equilibrate", type=int, default=3,
                    help="groups of 100 untimed FP64 steps (cancel_vcom + tnorm after each, md.F:87-101) "
                         "that bring every timed box to its run state before the warm-up steps")
    ap.add_argument("--drift-warmup", type=int, default=20,
                    help="warm-up groups of 100 steps (cancel_vcom + tnorm after each) before --drift")
    ap.add_argument("--ensemble-steps", type=int, default=100)
    ap.add_argument("--line-drift-steps", type=int, default=10000,
                    help="steps of the drift block of the default line (0: leave it out)")
    ap.add_argument("--no-served", action="store_true",
                    help="leave the served-ensemble block out of the default line")
    ap.add_argument("--served-rate", type=float, default=64.0,
                    help="Poisson arrival rate (runs/s) of the served ensemble in the default line")
    ap.add_argument("--serve", action="store_true",
                    help="instead of the benchmark: serve a request stream and report latency")
    ap.add_argument("--tune-report", action="store_true",
                    help="instead of the benchmark: run the autotuner on the pure-ion OCP (N=4,096), the ion "
                         "mixture (N=55,296), nucleons (N=51,200) and the 256-replica ensemble and report the "
                         "candidates tried and the winners")
    ap.add_argument("--serve-ensemble", action="store_true",
                    help="instead of the benchmark: serve the 256-replica ensemble and report latency")
    ap.add_argument("--ensemble-serve-steps", type=int, default=1000)
    ap.add_argument("--serve-count", type=int, default=48)
    ap.add_argument("--serve-rate", type=float, default=8.0)
    ap.add_argument("--serve-nmax", type=int, default=32768)
    ap.add_argument("--serve-smax", type=int, default=1000)
    return ap.parse_args()


def make_workload(kind, seed, n=0):
    from yukawamd_b200 import configs
    kw = {"n": n} if n else {}
    if kind == "mix":
        return configs.ion_mixture_cfg(seed, **kw)
    if kind == "ocp":
        return configs.pure_ion_ocp(seed, **kw)
    return configs.nucleon_matter(seed, **kw)


def equilibrate(w, groups, dist):
    """The workload with its positions and velocities after md.F's warm-up
    (`groups` groups of 100 FP64 steps, each followed by cancel_vcom and
    tnorm, md.F:87-101): the state a long run spends its steps in.  The
    uniform random start has pairs closer than the liquid allows, and timing
    its first steps would time a box that is not yet the run's."""
    if groups <= 0:
        return w
    import dataclasses
    from yukawamd_b200 import abi
    from yukawamd_b200.driver import RunControl, run_md
    from yukawamd_b200.engine import Engine
    with Engine(w, device=dist.local, precision=abi.YK_PREC_FP64) as e:
        run_md(e, RunControl(nwgroup=groups, nwsteps=100))
        x, v, _vold, _a = e.get_state()
    return dataclasses.replace(w, x=np.ascontiguousarray(x), v=np.ascontiguousarray(v))


def workload_desc(w, kind):
    n = w.n
    if kind == "mix":
        return ("ion-mixture N=%d Z={6,8,26} fractions {0.2,0.7,0.1} A=2Z n=7.18e-5/fm^3 "
                "kappa=0.5 Gamma_eff=150 (int_ion_mix.f)" % n)
    if kind == "ocp":
        return "pure-ion OCP N=%d Z=8 A=16 kappa=1 Gamma=175 (int_ion_pure.f)" % n
    return "nucleon N=%d x_p=0.4 n_B=0.05/fm^3 kT=1 HPP + p-p Coulomb lambda=10 (int_nn.f)" % n


# ---------------------------------------------------------------------------
# distributed plumbing (torch.distributed for barriers and the max over ranks)

class Dist:
    """One process per GPU (torchrun env vars).  NCCL on GPUs; gloo when no GPU
    is visible (the CPU tests of this plumbing).  Every rank makes the same
    collective calls in the same order; the process group has a short timeout
    so that a rank that never arrives ends the others' next collective with
    an error instead of a hang."""

    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = False
        self.torch = None
        self.dev = "cpu"

    def init(self, backend=None, timeout_s=120):
        if self.world > 1:
            import datetime
            import torch
            import torch.distributed as dist
            if backend is None:
                backend = "nccl" if torch.cuda.is_available() else "gloo"
            kw = {}
            if backend == "nccl":
                torch.cuda.set_device(self.local)
                self.dev = "cuda"
                kw["device_id"] = torch.device("cuda", self.local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
            self.torch = torch
            self.pg = True

    def barrier(self):
        if self.pg:
            t = self.torch.ones(1, device=self.dev)
            self.torch.distributed.all_reduce(t)
            if self.dev == "cuda":
                self.torch.cuda.synchronize()

    def _reduce(self, x, op):
        t = self.torch.tensor([float(x)], device=self.dev, dtype=self.torch.float64)
        self.torch.distributed.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x):
        if not self.pg:
            return x
        return self._reduce(x, self.torch.distributed.ReduceOp.MAX)

    def sum(self, x):
        if not self.pg:
            return x
        return self._reduce(x, self.torch.distributed.ReduceOp.SUM)

    def close(self):
        if self.pg:
            self.torch.distributed.destroy_process_group()
            self.pg = False


def job_rate(world, units_per_rank, ms_max):
    """Whole-job throughput of `world` replicas that each processed
    units_per_rank units, timed as the slowest rank (ms)."""
    return world * units_per_rank / (ms_max * 1e-3)


# ---------------------------------------------------------------------------
# clocks during the timed region

class ClockSampler:
    FIELDS = ("uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid):
        self.uuid = uuid
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        time.sleep(0.25)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, smax, reasons = [], None, set()
        for line in self.lines:
            f = [t.strip() for t in line.split(",")]
            if len(f) < 8:
                continue
            if self.uuid and self.uuid not in f[0]:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for name, val in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                                  "sw_power_cap"), f[4:8]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


class NvmlClockSampler:
    """SM clock and clock-event reasons of one GPU read through NVML every
    `period_s` from a host thread, started and stopped around the timed steps
    only, so that every sample falls inside the timed region (nvidia-smi's
    shortest period is longer than a whole 20-step run).  Read-only queries."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))

    def __init__(self, uuid, period_s=0.002):
        import pynvml
        self.nv = pynvml
        pynvml.nvmlInit()
        self.h = None
        # torch reports the UUID without NVML's "GPU-" prefix: match by substring
        for k in range(pynvml.nvmlDeviceGetCount()):
            hk = pynvml.nvmlDeviceGetHandleByIndex(k)
            u = pynvml.nvmlDeviceGetUUID(hk)
            u = u.decode() if isinstance(u, bytes) else u
            if uuid and uuid in u:
                self.h = hk
                break
        if self.h is None:
            raise RuntimeError("no NVML device with UUID %s" % uuid)
        self.period = period_s
        self.samples = []
        self.bits = 0
        self._stop = threading.Event()
        self.thread = None

    def _poll(self):
        nv = self.nv
        read_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            nv.nvmlDeviceGetCurrentClocksThrottleReasons
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
                self.bits |= int(read_reasons(self.h))
            except nv.NVMLError:
                pass
            time.sleep(self.period)

    def start(self):
        self._stop.clear()
        self.thread = threading.Thread(target=self._poll, daemon=True)
        self.thread.start()

    def stop(self):
        self._stop.set()
        if self.thread:
            self.thread.join(timeout=2)

    def result(self):
        nv = self.nv
        if not self.samples:
            return None
        smax = nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM)
        reasons = sorted(name for name, const in self.REASONS if self.bits & int(getattr(nv, const, 0)))
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": float(smax), "reasons": reasons,
                "samples": len(self.samples), "sampler": "NVML every %.0f ms during the timed steps"
                                                         % (1e3 * self.period)}


def device_uuid(dev):
    try:
        import torch
        return str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        return None


# ---------------------------------------------------------------------------
# our arm

KERNEL_CHOICE = [0]       # --kernel: 0 auto, 1 rows, 2 pairs, 3 near lists


def time_engine(w, precision, steps, warmup, meas_every, dist, flush=True, sampler=None):
    """W untimed steps, then K timed steps; returns (ms_total, perf, launches)."""
    from yukawamd_b200 import abi
    from yukawamd_b200.engine import Engine, kernel_launch_count
    prec = abi.YK_PREC_MIXED if precision == "mixed" else abi.YK_PREC_FP64
    e = Engine(w, precision=prec, device=dist.local)
    if KERNEL_CHOICE[0]:
        e.set_tuning(force_kernel=KERNEL_CHOICE[0])
    t = e.tuning()
    e.kernel_name = {1: "k_force_rows", 2: "k_force_pairs", 3: "k_force_near"}.get(t.force_kernel, "?")
    if t.force_kernel == 2 and t.targets_per_thread == 2:
        e.kernel_name = "k_force_pairs2"
    e.accel(True)                                  # md.F:69, initial forces
    if warmup:
        e.run(warmup, meas_every, series=False)
    e.perf_enable(True, L2_FLUSH_BYTES if flush else 0)
    dist.barrier()
    l0 = kernel_launch_count()
    if sampler is not None:
        sampler.start()
    e.run(steps, meas_every, series=False)
    if sampler is not None:
        sampler.stop()
    launches = kernel_launch_count() - l0
    dist.barrier()
    perf = e.perf_read()
    e.perf_enable(False, 0)
    return e, perf, launches


def e2e_engine(w, steps, warmup, meas_every, dist):
    """Public-API loop with host buffers: every step copies x and v from
    page-locked host memory to the device, runs newton, and copies x, v back
    (the sync the Fortran shim makes while the driver keeps host-side tnorm /
    cancel_vcom / strain)."""
    from yukawamd_b200.engine import Engine, host_register, host_unregister
    e = Engine(w, device=dist.local)
    e.accel(True)
    x = np.ascontiguousarray(w.x.copy())
    v = np.ascontiguousarray(w.v.copy())
    host_register(x)
    host_register(v)
    try:
        for s in range(warmup):
            e.set_state(x=x, v=v)
            e.newton((s + 1) % meas_every == 0 if meas_every else False)
            e.get_into(x=x, v=v)
        dist.barrier()
        t0 = time.perf_counter()
        for s in range(steps):
            e.set_state(x=x, v=v)
            sc = e.newton((s + 1) % meas_every == 0 if meas_every else False)
            e.get_into(x=x, v=v)
            _ = sc.ev
        t1 = time.perf_counter()
        dist.barrier()
    finally:
        host_unregister(x)
        host_unregister(v)
        e.close()
    return (t1 - t0) * 1e3, 2 * 24 * w.n, 2 * 24 * w.n + 112


def read_traffic(kind, precision):
    """DRAM bytes per force launch from the committed ncu summaries
    (a line "traffic_bytes_per_launch <kind> <precision>: <bytes>")."""
    key = "traffic_bytes_per_launch %s %s:" % (kind, precision)
    pdir = os.path.join(ROOT, "profiles")
    if not os.path.isdir(pdir):
        return None
    for name in sorted(os.listdir(pdir)):
        if not name.endswith(".md"):
            continue
        for line in open(os.path.join(pdir, name)):
            if line.startswith(key):
                try:
                    return float(line.split(":", 1)[1].split()[0])
                except ValueError:
                    return None
    return None


def read_pipe(kind, precision):
    """Busy share of the bounding pipe of the force kernel in one ncu capture
    (a line "pipe_pct_per_launch <kind> <precision>: <pct> <pipe>" in the
    committed ncu summaries), as {"pipe", "pct"}; None if absent."""
    key = "pipe_pct_per_launch %s %s:" % (kind, precision)
    pdir = os.path.join(ROOT, "profiles")
    if not os.path.isdir(pdir):
        return None
    for name in sorted(os.listdir(pdir)):
        if not name.endswith(".md"):
            continue
        for line in open(os.path.join(pdir, name)):
            if line.startswith(key):
                f = line.split(":", 1)[1].split()
                try:
                    return {"pipe": f[1], "pct": float(f[0]), "source": "profiles/" + name}
                except (ValueError, IndexError):
                    return None
    return None


def _pairs_of_rows(n, r0, r1):
    """Unique pairs of target rows r0 <= i < r1 (row i pairs with j > i)."""
    r1 = min(r1, n - 1)
    if r1 <= r0:
        return 0
    return (r1 - r0) * (n - 1) - (r0 + r1 - 1) * (r1 - r0) // 2


def cpu_rows(n, rate, budget_s):
    """Target rows for one timed CPU call: all of them when a whole force
    call fits budget_s at `rate` pairs/s, else a block centred on the middle
    row.  The reference's loop costs a per-row part (its omp for / omp single
    barriers, int_ion_mix.f:159-213) plus a part proportional to the row's
    n-1-i pairs; a centred block has the whole call's mean row length, so
    both parts weigh as in a whole call."""
    total = n * (n - 1) // 2
    if total <= budget_s * rate:
        return 0, n, "whole force calls over"
    # rows of mean length (n-1)/2 cost about (n-1)/2 pairs each
    nrows = int(min(n - 2, max(64, 2.0 * budget_s * rate / (n - 1))))
    r0 = max(0, (n - nrows) // 2)
    return r0, r0 + nrows, "target rows %d..%d (centred on the middle row) of" % (r0, r0 + nrows)


def _calibrate(orc, p, w):
    """pairs/s of the oracle's OpenMP loop on a small centred block."""
    n = w.n
    r0 = max(0, n // 2 - 32)
    orc.set_row_range(r0, r0 + 64)
    t0 = time.perf_counter()
    orc.accel(p, w.x, w.zii, w.aii, False)
    dt = time.perf_counter() - t0
    orc.set_row_range()
    return _pairs_of_rows(n, r0, r0 + 64) / max(dt, 1e-6)


def cpu_sample(w, kind, target_s=12.0):
    """Time the oracle's OpenMP force loop (reference structure) on all host
    cores: whole force calls repeated to about target_s, or one centred block
    of target rows when a whole call takes longer."""
    from oracle.oracle import Oracle
    cores = os.cpu_count() or 1
    orc = Oracle("double", threads=cores)
    p = w.yk_params()
    n = w.n
    rate = _calibrate(orc, p, w)
    r0, r1, what = cpu_rows(n, rate, target_s)
    pairs1 = _pairs_of_rows(n, r0, r1)
    reps = max(1, int(round(target_s * rate / max(pairs1, 1))))
    orc.set_row_range(r0, r1)
    t0 = time.perf_counter()
    for _ in range(reps):
        orc.accel(p, w.x, w.zii, w.aii, False)
    dt = time.perf_counter() - t0
    orc.set_row_range()
    pairs = reps * pairs1
    return {"value": pairs / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": "force-only calls of the oracle's OpenMP loop (%s structure, OMP_SCHEDULE=%s): "
                      "%d calls, %s the full N=%d box, %d pairs in %.2f s"
                      % ({"mix": "int_ion_mix.f", "ocp": "int_ion_pure.f"}.get(kind, "int_nn.f"),
                         os.environ.get("OMP_SCHEDULE", "static"), reps, what, n, pairs, dt)}


def run_ours(args, dist):
    from yukawamd_b200 import _lib
    from yukawamd_b200.engine import peak_probe
    kind = args.workload
    w0 = make_workload(kind, args.seed + dist.rank, args.n)
    w = equilibrate(w0, args.equilibrate, dist)
    pairs_step = w.pairs_per_step
    K, W, me = args.steps, args.warmup, args.meas_every

    uuid = device_uuid(dist.local)
    try:
        nvs = NvmlClockSampler(uuid)
    except Exception:
        nvs = None
    if nvs is None:
        clocks = ClockSampler(uuid)
        clocks.start()
    e, perf, launches = time_engine(w, args.precision, K, W, me, dist, sampler=nvs)
    clk = nvs.result() if nvs is not None else clocks.stop()
    ms_local = perf.run_ms
    ms = dist.max(ms_local)
    value = job_rate(dist.world, pairs_step * K, ms)

    # dominant kernel: the force kernel, timed live with events on its stream
    force_ms = perf.force_ms / max(perf.force_calls, 1)
    meas_frac = (K // me) / K if me else 0.0
    fpp = (1 - meas_frac) * FLOPS_PER_PAIR[(kind, False)] + meas_frac * FLOPS_PER_PAIR[(kind, True)]
    prec_kind = 1 if args.precision == "mixed" else 0
    peak = peak_probe(dist.local, prec_kind)
    achieved = fpp * pairs_step / (force_ms * 1e-3) / 1e12
    roofline = {"bound": "fp64" if prec_kind == 0 else "fp32", "achieved": achieved,
                "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "traffic": read_traffic(kind, args.precision),
                "kernel": "%s + k_combine (force call), avg %.3f ms/launch over %d launches"
                          % (e.kernel_name, force_ms, perf.force_calls),
                "peak_source": "measured live by yk_peak_probe (%s FMA chain, all SMs)"
                               % ("FP64" if prec_kind == 0 else "FP32"),
                "flops_per_pair": fpp, "force_share_of_step": perf.force_ms / perf.run_ms,
                "pipe_ncu": read_pipe(kind, args.precision),
                "note": "achieved counts flops_per_pair on every unique pair; the pipe_ncu busy share "
                        "is what the hardware pipe did"}

    out = {"metric": HEADLINE_METRIC, "value": value, "unit": UNIT, "n_gpus": dist.world,
           "steps": K, "warmup": W, "ms_per_step": ms / K, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None,
           "dtype": "f64" if args.precision == "fp64" else "f64+f32",
           "data": "synthetic: numpy PCG64 seed %d (+rank), uniform positions, Maxwell "
                   "velocities with zero momentum, then %d untimed groups of 100 FP64 steps with "
                   "cancel_vcom + tnorm (md.F warm-up)" % (args.seed, args.equilibrate),
           "config": {"workload": workload_desc(w, kind), "n": w.n,
                      "pairs_per_step": pairs_step, "precision": args.precision,
                      "integrator": "vel_verlet_2", "meas_every": me,
                      "l2": "flushed: 256 MiB device memset between timed steps (each step "
                            "timed by its own CUDA-event pair after the flush)",
                      "parallelism": "replicas x%d (one box per GPU, no collective)" % dist.world},
           "roofline": roofline, "gpu_launches": launches, "clocks": clk}
    e.close()

    if not args.no_companion:
        other = "mixed" if args.precision == "fp64" else "fp64"
        e2, perf2, _ = time_engine(w, other, K, W, me, dist)
        ms2 = dist.max(perf2.run_ms)
        v2 = job_rate(dist.world, pairs_step * K, ms2)
        # force accuracy of the mixed form against FP64 on the same positions
        from yukawamd_b200 import abi
        from yukawamd_b200.engine import Engine
        with Engine(w, device=dist.local) as a64, \
                Engine(w, device=dist.local, precision=abi.YK_PREC_MIXED) as a32:
            s64 = a64.accel(True)
            s32 = a32.accel(True)
            n = w.n
            ferr = float(np.linalg.norm(a32.a[:3 * n] - a64.a[:3 * n]) /
                         np.linalg.norm(a64.a[:3 * n]))
            ev_err = abs(s32.ev - s64.ev) / abs(s64.ev)
            px_err = abs(s32.px - s64.px) / abs(s64.px)
        out[other] = {"value": v2, "ms_per_step": ms2 / K,
                      "ratio_mixed_over_fp64": (v2 / value) if other == "mixed" else (value / v2),
                      "force_rms_rel_err_vs_fp64": ferr, "ev_rel_err": ev_err,
                      "px_rel_err": px_err}
        # the companion's force kernel against its own pipe's measured peak
        kind2 = 1 if other == "mixed" else 0
        fms2 = perf2.force_ms / max(perf2.force_calls, 1)
        ach2 = fpp * pairs_step / (fms2 * 1e-3) / 1e12
        peak2 = peak_probe(dist.local, kind2)
        out[other]["roofline"] = {"bound": "fp32" if kind2 else "fp64", "achieved": ach2, "peak": peak2,
                                  "unit": "TFLOP/s", "frac": ach2 / peak2,
                                  "traffic": read_traffic(kind, other),
                                  "kernel": "%s + k_combine (force call), avg %.3f ms/launch over %d launches"
                                            % (e2.kernel_name, fms2, perf2.force_calls),
                                  "peak_source": "measured live by yk_peak_probe (%s FMA chain, all SMs)"
                                                 % ("FP32" if kind2 else "FP64"),
                                  "flops_per_pair": fpp, "pipe_ncu": read_pipe(kind, other)}
        e2.close()
        if dist.rank == 0 and dist.world == 1 and not args.no_cpu:
            out["mixed"]["vs_oracle"] = mixed_vs_oracle(w)

    if not args.no_extras and dist.world == 1:
        out["nucleon"] = nucleon_pair(K, W, me, dist, args.equilibrate)
        out["ensemble"] = ensemble(args.ensemble_steps, me, dist)
        if args.line_drift_steps > 0:
            out["drift"] = drift_block(w0, kind, args.line_drift_steps, args.drift_warmup, dist)
        if not args.no_served:
            out["served"] = served_ensemble(args, dist)

    if not args.no_e2e:
        t_e2e, bi, bo = e2e_engine(w, K, W, me, dist)
        t_e2e = dist.max(t_e2e)
        out["e2e"] = {"value": dist.world * pairs_step * K / (t_e2e * 1e-3), "unit": UNIT,
                      "h2d_bytes_per_step": bi, "d2h_bytes_per_step": bo,
                      "ms_per_step": t_e2e / K,
                      "path": "Engine.set_state(x,v) -> Engine.newton -> Engine.get_into(x,v), "
                              "page-locked host buffers, wall clock"}

    if dist.rank == 0 and dist.world == 1 and not args.no_cpu:
        out["cpu_baseline"] = cpu_sample(w, kind)
    return out


def mixed_vs_oracle(w):
    """The mixed form's errors against one complete call of the FP64 CPU oracle
    (int_ion_mix.f:105-295 restated, OpenMP on all host cores) on the same
    positions: force 2-norm relative error, ev, px and pp."""
    from oracle.oracle import Oracle
    from yukawamd_b200 import abi
    from yukawamd_b200.engine import Engine
    orc = Oracle("double", threads=os.cpu_count() or 1)
    p = w.yk_params()
    n = w.n
    t0 = time.perf_counter()
    a_ref, s_ref = orc.accel(p, w.x, w.zii, w.aii, True)
    t_orc = time.perf_counter() - t0
    with Engine(w, precision=abi.YK_PREC_MIXED) as e:
        s = e.accel(True)
        a = e.a.copy()
    return {"force_rms_rel_err": float(np.linalg.norm(a[:3 * n] - a_ref[:3 * n]) / np.linalg.norm(a_ref[:3 * n])),
            "ev_rel_err": abs(s.ev - s_ref.ev) / abs(s_ref.ev),
            "px_rel_err": abs(s.px - s_ref.px) / abs(s_ref.px),
            "pp_rel_err": float(np.linalg.norm(np.array(s.pp) - np.array(s_ref.pp)) / np.linalg.norm(np.array(s_ref.pp))),
            "oracle": "one measuring force call of the FP64 CPU oracle over all N(N-1)/2 pairs (%.1f s, %d threads)"
                      % (t_orc, os.cpu_count() or 1)}


def drift_block(w, kind, steps, warmup_groups, dist):
    """Total-energy drift of the benchmark box over `steps` steps in FP64 and
    in the mixed form, from one state equilibrated as md.F does (warm-up
    groups of 100 FP64 steps, each followed by cancel_vcom and tnorm,
    md.F:87-101); E = ev + ek per particle every 100 steps (the cadence of
    md.F's energy record, md.F:125-157)."""
    from yukawamd_b200 import abi
    from yukawamd_b200.driver import RunControl, run_md
    from yukawamd_b200.engine import Engine
    out = {"workload": workload_desc(w, kind), "steps": steps, "every": 100,
           "warmup": "%d groups x 100 FP64 steps with cancel_vcom + tnorm (md.F:87-101)" % warmup_groups}
    x, v = w.x, w.v
    t0 = time.perf_counter()
    if warmup_groups > 0:
        with Engine(w, device=dist.local, precision=abi.YK_PREC_FP64) as e:
            run_md(e, RunControl(nwgroup=warmup_groups, nwsteps=100))
            x, v, _vold, _a = e.get_state()
    for prec in ("fp64", "mixed"):
        yp = w.yk_params(precision=abi.YK_PREC_MIXED if prec == "mixed" else abi.YK_PREC_FP64)
        with Engine(yp, x, v, w.zii, w.aii, device=dist.local) as e:
            s0 = e.accel(True)
            e0 = s0.ev + e.ttot()
            ser = e.run(steps, 100)
            es = np.array([ser[k].ev + ser[k].ek for k in range(99, steps, 100)])
        out[prec] = {"E0": e0, "max_abs_dE_over_E": float(np.max(np.abs(es - e0)) / abs(e0)),
                     "end_dE_over_E": float((es[-1] - e0) / abs(e0))}
    out["target"] = "max |dE/E| <= 1e-5"
    out["wall_s"] = time.perf_counter() - t0
    return out


def served_ensemble(args, dist):
    """The 256-replica ensemble (256 pure-ion boxes, N log-uniform in
    [1e3, 2e4], Gamma U[50, 250], kappa U[0.5, 2], Z in {6, 8, 26}, 1,000 steps
    each, mixed precision) served with Poisson arrivals: p50 / p99 completion
    latency and aggregate pair-interactions/s."""
    from yukawamd_b200 import abi, configs
    from yukawamd_b200.serve import Request, Server
    seed = args.seed + 2 + 1000 * dist.rank
    boxes = configs.replica_ensemble(seed)
    rng = np.random.default_rng(np.random.PCG64(seed + 77))
    arrivals = np.cumsum(rng.exponential(1.0 / args.served_rate, len(boxes)))
    arrivals -= arrivals[0]
    reqs = [Request(i, w, args.ensemble_serve_steps, abi.YK_PREC_MIXED, float(t))
            for i, (w, t) in enumerate(zip(boxes, arrivals))]
    rep = Server(device=dist.local, chunk=50).run(reqs)
    rep.pop("fp64_shadows", None)
    rep["stream"] = ("256 pure-ion boxes, N log-uniform in [1e3, 2e4], Gamma U[50,250], kappa U[0.5,2], "
                     "Z in {6,8,26}, seed %d, %d steps each, mixed precision, Poisson arrivals at %.0f runs/s "
                     "(the last at %.2f s)" % (seed, args.ensemble_serve_steps, args.served_rate, arrivals[-1]))
    return rep


def nucleon_pair(K, W, me, dist, groups=0):
    """int_nn.f at N = 51,200 (proton fraction 0.4, n_B = 0.05 fm^-3, kT = 1
    MeV): FP64 and mixed pairs/s and the mixed form's accuracy, from the state
    after `groups` md.F warm-up groups."""
    from yukawamd_b200 import abi
    from yukawamd_b200.engine import Engine
    w = equilibrate(make_workload("nucleon", 3 + dist.rank), groups, dist)
    res = {"workload": workload_desc(w, "nucleon"), "pairs_per_step": w.pairs_per_step}
    for prec in ("fp64", "mixed"):
        e, perf, _ = time_engine(w, prec, K, W, me, dist)
        res[prec] = {"value": w.pairs_per_step * K / (dist.max(perf.run_ms) * 1e-3),
                     "ms_per_step": perf.run_ms / K}
        e.close()
    res["ratio_mixed_over_fp64"] = res["mixed"]["value"] / res["fp64"]["value"]
    with Engine(w, device=dist.local) as a64, \
            Engine(w, device=dist.local, precision=abi.YK_PREC_MIXED) as a32:
        s64 = a64.accel(True)
        s32 = a32.accel(True)
        n = w.n
        res["force_rms_rel_err_vs_fp64"] = float(np.linalg.norm(a32.a[:3 * n] - a64.a[:3 * n]) /
                                                 np.linalg.norm(a64.a[:3 * n]))
        res["ev_rel_err"] = abs(s32.ev - s64.ev) / abs(s64.ev)
    if dist.rank == 0 and dist.world == 1:
        res["mixed_vs_oracle"] = mixed_vs_oracle(w)
    return res


def ensemble(steps, me, dist, precision="mixed", seed=4):
    """The replica ensemble: 256 pure-ion boxes, N log-uniform in
    [1e3, 2e4], Gamma U[50,250], kappa U[0.5,2], Z in {6,8,26}, advanced
    together by the batch engine (CUDA graphs of 50 steps)."""
    from yukawamd_b200 import abi, configs
    from yukawamd_b200.engine import Batch
    boxes = configs.replica_ensemble(seed + 1000 * dist.rank)
    prec = abi.YK_PREC_MIXED if precision == "mixed" else abi.YK_PREC_FP64
    pairs = sum(w.pairs_per_step for w in boxes)
    with Batch(boxes, device=dist.local, precision=prec) as b:
        b.accel(True)
        b.run(50, me, series=False)                 # warm-up (one graph)
        dist.barrier()
        _, ms = b.run(steps, me, series=False)
        dist.barrier()
    ms = dist.max(ms)
    return {"workload": "%d pure-ion boxes, N log-uniform in [1000, 20000] (sum %d), Gamma U[50,250], "
                        "kappa U[0.5,2], Z in {6,8,26}; seed %d" % (len(boxes), sum(w.n for w in boxes), seed),
            "precision": precision, "steps": steps, "graph_steps": 50,
            "pairs_per_step": pairs, "value": dist.world * pairs * steps / (ms * 1e-3),
            "ms_per_step": ms / steps}


def drift(args, dist):
    """--drift N: the drift block alone, for N steps of the chosen workload."""
    w = make_workload(args.workload, args.seed, args.n)
    return drift_block(w, args.workload, args.drift, args.drift_warmup, dist)


def serve_stream(args, dist):
    """The served request stream: Poisson arrivals, 70 % ion (pure or mixture)
    and 30 % nucleon runs, N log-uniform in [512, nmax], steps uniform in
    [100, smax], mixed precision with an FP64 twin for 1 run in 16."""
    from yukawamd_b200 import configs
    from yukawamd_b200.serve import Server, make_requests
    stream = configs.request_stream(seed=args.seed, count=args.serve_count, rate_per_s=args.serve_rate,
                                    nmin=512, nmax=args.serve_nmax, smin=100, smax=args.serve_smax)
    reqs = make_requests(stream, shadow_every=16)
    srv = Server(device=dist.local, chunk=50)
    rep = srv.run(reqs)
    rep.update({"metric": "served p99 completion latency; aggregate pair-interactions/s",
                "stream": "%d runs, Poisson rate %.2f/s, 70%% ion / 30%% nucleon, N log-uniform in "
                          "[512, %d], steps U[100, %d], mixed precision, FP64 twin 1 in 16, seed %d"
                          % (args.serve_count, args.serve_rate, args.serve_nmax, args.serve_smax, args.seed)})
    return rep


def serve_ensemble(args, dist):
    """The 256-replica ensemble served: every replica is a request of
    args.ensemble_serve_steps steps submitted at t = 0; the server keeps them
    resident and advances them as one batch (one persistent force kernel per
    step, CUDA graphs of 50 steps) with the job segment length the autotuner
    picked on this ensemble.  Reports p50 / p99 completion latency and the
    aggregate pair-interactions/s."""
    from yukawamd_b200 import abi, configs, tune
    from yukawamd_b200.engine import Batch
    from yukawamd_b200.serve import Request, Server
    boxes = configs.replica_ensemble(args.seed + 2 + 1000 * dist.rank)
    t0 = time.perf_counter()
    with Batch(boxes, device=dist.local, precision=abi.YK_PREC_MIXED) as b:
        b.accel(True)
        best, best_ms, tried = tune.tune_batch(b, steps=50, device=dist.local)
    tune_s = time.perf_counter() - t0
    reqs = [Request(i, w, args.ensemble_serve_steps, abi.YK_PREC_MIXED, 0.0) for i, w in enumerate(boxes)]
    rep = Server(device=dist.local, chunk=50, autotune=True).run(reqs)
    rep.update({"metric": "served 256-replica ensemble: p50 / p99 completion latency; aggregate "
                          "pair-interactions/s",
                "ensemble": "256 pure-ion boxes, N log-uniform in [1e3, 2e4], Gamma U[50,250], kappa "
                            "U[0.5,2], Z in {6,8,26}, seed %d, %d steps each, all submitted at t = 0, "
                            "mixed precision" % (args.seed + 2 + 1000 * dist.rank, args.ensemble_serve_steps),
                "autotune": {"pair_seg": best, "graph_ms_50_steps": best_ms,
                             "tried": [[ms, seg] for ms, seg in tried], "wall_s": tune_s}})
    return rep


def tune_report(args, dist):
    """The autotuner (yukawamd_b200/tune.py) on the benchmark workloads: for
    each single box every candidate's step and force-call times (CUDA events,
    16 steps) and the winner (shortest step); for the replica ensemble every
    job segment length's graph time."""
    from yukawamd_b200 import abi, configs, tune
    from yukawamd_b200.engine import Batch, Engine
    out = {"metric": "autotuner: step ms and force-call ms per candidate (single boxes), graph ms per 50 steps "
                     "(ensemble)"}
    for name, w in (("ocp_4096", configs.pure_ion_ocp(1)), ("mix_55296", configs.ion_mixture_cfg(2)),
                    ("nucleon_51200", configs.nucleon_matter(3))):
        for prec in ("fp64", "mixed"):
            p = abi.YK_PREC_MIXED if prec == "mixed" else abi.YK_PREC_FP64
            with Engine(w, device=dist.local, precision=p) as e:
                e.accel(True)
                best, best_ms, res = tune.tune(e, device=dist.local, save=False)
            out["%s_%s" % (name, prec)] = {
                "winner": best, "step_ms": best_ms,
                "tried": [[r[0] if r[0] != float("inf") else None, r[1],
                           r[3] if r[3] != float("inf") else None] for r in res]}
    boxes = configs.replica_ensemble(4)
    with Batch(boxes, device=dist.local, precision=abi.YK_PREC_MIXED) as b:
        b.accel(True)
        best, best_ms, tried = tune.tune_batch(b, steps=50, device=dist.local, save=False)
    out["ensemble_256_mixed"] = {"winner": {"pair_seg": best}, "graph_ms_50_steps": best_ms,
                                 "tried": [[ms, {"pair_seg": seg}] for ms, seg in tried]}
    return out


def run_reference(args):
    """The reference's CPU algorithm (OpenMP C restatement) on all host cores."""
    from oracle.oracle import Oracle
    kind = args.workload
    w = make_workload(kind, args.seed, args.n)
    n = w.n
    p = w.yk_params()
    cores = os.cpu_count() or 1
    orc = Oracle("double", threads=cores)
    # each step is one force call over whole box when that takes <= 4 s on
    # these cores, else over a centred block of rows of about 4 s, so the
    # whole --steps K --warmup W run stays within minutes
    rate = _calibrate(orc, p, w)
    r0, r1, what = cpu_rows(n, rate, 4.0)
    orc.set_row_range(r0, r1)
    for _ in range(args.warmup):
        orc.accel(p, w.x, w.zii, w.aii, False)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        orc.accel(p, w.x, w.zii, w.aii, False)
        times.append(time.perf_counter() - t0)
    orc.set_row_range()
    pairs = _pairs_of_rows(n, r0, r1)
    total = sum(times)
    value = pairs * args.steps / total
    sample = ("each step: one force-only call of the oracle's OpenMP loop (reference "
              "structure: omp for over j per target i, omp single fold; OMP_SCHEDULE=%s) over %s "
              "the full N=%d box = %d pairs" % (os.environ.get("OMP_SCHEDULE", "static"), what, n, pairs))
    return {"metric": HEADLINE_METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: numpy PCG64 seed %d" % args.seed, "impl": "reference",
            "config": {"workload": workload_desc(w, kind), "n": n, "precision": "fp64",
                       "parallelism": "OpenMP %d threads" % cores},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def main():
    args = parse()
    if args.impl == "reference":
        if int(os.environ.get("RANK", "0")) != 0:
            return 0
        print(json.dumps(run_reference(args)), flush=True)
        return 0
    KERNEL_CHOICE[0] = {"auto": 0, "rows": 1, "pairs": 2, "near": 3}[args.kernel]
    dist = Dist()
    dist.init()
    try:
        if args.tune_report:
            out = tune_report(args, dist)
            if dist.rank == 0:
                print(json.dumps(out), flush=True)
            return 0
        if args.serve_ensemble:
            out = serve_ensemble(args, dist)
            if dist.rank == 0:
                print(json.dumps(out), flush=True)
            return 0
        if args.serve:
            out = serve_stream(args, dist)
            if dist.rank == 0:
                print(json.dumps(out), flush=True)
            return 0
        if args.drift:
            out = drift(args, dist)
            if dist.rank == 0:
                print(json.dumps(out), flush=True)
            return 0
        out = run_ours(args, dist)
        if dist.rank == 0:
            print(json.dumps(out), flush=True)
    finally:
        dist.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
