"""Autotuner for the engine's tunables.

For one box the engine can run its force call three ways (the half-pair
kernel with scratch, the same over per-warp near-source lists, or the row
kernel that evaluates each pair from both sides), cap the half-pair jobs at
`pair_seg` source tiles (the job list shrinks them towards its end), let
1, 2 or 4 CTAs share each 128-target block (`source_split`: the threads per
target, for small boxes), give each thread one or two targets
(`targets_per_thread`: target blocks of 128 or 256 slots, the tile shape of
the ion kernels); it refreshes
the Hilbert order every `sort_every` steps.  Which choice is fastest depends on
N, the cutoff radius relative to the box, the interaction and the precision,
so the tuner measures candidates on the caller's own workload (CUDA-event
time per step, sorts included, yk_perf, over a window of 16 steps: the force
call slows down step by step after a sort as particles leave their
neighbours, which a shorter window would not see) and remembers the winner per

    (GPU name, sim type, precision, N bucket)      N bucket = round(2 log2 N)

in a JSON cache (default ~/.cache/yukawamd_b200/tune.json, or $YK_TUNE_CACHE).
Engine.autotune() / tune.apply(engine) use it transparently.
"""
import json
import math
import os
import time

from . import abi

# sort_every 0 is the engine's automatic cadence (4 steps)
CANDIDATES = [
    dict(force_kernel=abi.KERNEL_NEAR, pair_seg=8, sort_every=0),
    dict(force_kernel=abi.KERNEL_NEAR, pair_seg=4, sort_every=0),
    dict(force_kernel=abi.KERNEL_NEAR, pair_seg=16, sort_every=0),
    dict(force_kernel=abi.KERNEL_PAIRS, pair_seg=8, sort_every=0),
    dict(force_kernel=abi.KERNEL_PAIRS, pair_seg=4, sort_every=0),
    dict(force_kernel=abi.KERNEL_PAIRS, pair_seg=16, sort_every=0),
    dict(force_kernel=abi.KERNEL_PAIRS, pair_seg=2, sort_every=0),
    # re-sort cadence
    dict(force_kernel=abi.KERNEL_PAIRS, pair_seg=8, sort_every=2),
    dict(force_kernel=abi.KERNEL_PAIRS, pair_seg=8, sort_every=8),
    dict(force_kernel=abi.KERNEL_PAIRS, pair_seg=8, sort_every=16),
    dict(force_kernel=abi.KERNEL_PAIRS, pair_seg=8, sort_every=-1),
    dict(force_kernel=abi.KERNEL_ROWS, pair_seg=8, sort_every=0),
    # threads per target: 2 or 4 CTAs share each 128-target block (small boxes)
    dict(force_kernel=abi.KERNEL_PAIRS, pair_seg=1, sort_every=0, source_split=2),
    dict(force_kernel=abi.KERNEL_PAIRS, pair_seg=1, sort_every=0, source_split=4),
    # tile shape: two targets per thread (256-target blocks; ion boxes on the
    # FP64 exact-image or mixed hi/lo path, others fall back to one)
    dict(force_kernel=abi.KERNEL_PAIRS, pair_seg=8, sort_every=0, targets_per_thread=2),
    dict(force_kernel=abi.KERNEL_PAIRS, pair_seg=4, sort_every=0, targets_per_thread=2),
    dict(force_kernel=abi.KERNEL_PAIRS, pair_seg=16, sort_every=0, targets_per_thread=2),
]
# source_split > 1 makes one job per unit and part: only worth trying while the
# box has few tiles (it is there to fill the GPU with a small box)
SPLIT_MAX_N = 16384


def cache_path():
    p = os.environ.get("YK_TUNE_CACHE")
    if p:
        return p
    base = os.environ.get("XDG_CACHE_HOME", os.path.join(os.path.expanduser("~"), ".cache"))
    return os.path.join(base, "yukawamd_b200", "tune.json")


def _load():
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(doc):
    path = cache_path()
    os.makedirs(os.path.dirname(path), exist_ok=True)
    tmp = path + ".tmp%d" % os.getpid()
    with open(tmp, "w") as f:
        json.dump(doc, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def gpu_name(device=0):
    try:
        import torch
        return torch.cuda.get_device_name(device)
    except Exception:
        return "cuda:%d" % device


def bucket(n):
    return int(round(2.0 * math.log2(max(n, 1))))


def key_for(engine, device=0):
    p = engine.params
    return "%s|sim%d|prec%d|nb%d" % (gpu_name(device), p.sim_type, p.precision, bucket(engine.n))


def measure(engine, cand, steps=16, warmup=2):
    """Mean CUDA-event times (ms) per step (sorts included) and per force call
    under candidate `cand`.  The engine's state advances by warmup + steps
    steps."""
    engine.set_tuning(**cand)
    engine.run(warmup, 0, series=False)
    engine.perf_enable(True, 0)
    engine.run(steps, 0, series=False)
    perf = engine.perf_read()
    engine.perf_enable(False, 0)
    return perf.run_ms / max(perf.steps, 1), perf.force_ms / max(perf.force_calls, 1)


def tune(engine, candidates=None, steps=16, warmup=2, device=0, save=True):
    """Time every candidate on this engine's workload; apply and return the
    one with the shortest step (the result's ms) and the list of (step ms,
    candidate, error or None, force-call ms).  The engine's positions are
    restored afterwards, so tuning does not advance the caller's
    trajectory."""
    candidates = candidates or [c for c in CANDIDATES
                                if c.get("source_split", 1) == 1 or engine.n <= SPLIT_MAX_N]
    x, v, vold, a = engine.get_state()
    results = []
    for cand in candidates:
        cand = dict(cand)
        cand.setdefault("source_split", 1)
        cand.setdefault("targets_per_thread", 1)
        try:
            ms, fms = measure(engine, cand, steps, warmup)
        except Exception as exc:          # e.g. scratch too large for this N
            results.append((float("inf"), cand, str(exc), float("inf")))
            continue
        results.append((ms, cand, None, fms))
        engine.set_state(x=x, v=v, vold=vold, a=a)
    best_ms, best, _, best_fms = min(results, key=lambda r: r[0])
    engine.set_tuning(**best)
    engine.set_state(x=x, v=v, vold=vold, a=a)
    if save:
        doc = _load()
        doc[key_for(engine, device)] = dict(best, step_ms=best_ms, force_ms=best_fms, when=time.time(),
                                            n=engine.n, tried=[(r[0], r[1]) for r in results])
        _store(doc)
    return best, best_ms, results


BATCH_SEGS = (8, 4, 16, 2, 32)


def batch_key(batch, device=0):
    import numpy as np
    p = batch.params[0]
    return "%s|batch|sim%d|prec%d|nrep%d|nb%d" % (gpu_name(device), p.sim_type, p.precision, batch.nrep,
                                                  bucket(int(np.sqrt(np.mean(np.square(batch.n))))))


def tune_batch(batch, segs=BATCH_SEGS, steps=50, device=0, save=True):
    """Time one graph of `steps` steps of the whole batch for every job
    segment length (source tiles per work item) and keep the fastest.  The
    boxes' states are restored afterwards.  Cached per (GPU, sim, precision,
    box count, RMS box size bucket)."""
    states = [batch.get_state(r) for r in range(batch.nrep)]
    results = []
    for seg in segs:
        batch.set_tuning(pair_seg=seg, graph_steps=steps)
        batch.run(steps, 0, series=False)                  # capture + warm
        _, ms = batch.run(steps, 0, series=False)
        results.append((ms, seg))
        for r, (x, v, vold, a) in enumerate(states):
            batch.set_state(r, x=x, v=v, vold=vold, a=a)
    best_ms, best = min(results)
    batch.set_tuning(pair_seg=best, graph_steps=steps)
    if save:
        doc = _load()
        doc[batch_key(batch, device)] = dict(pair_seg=best, graph_steps=steps, ms=best_ms, when=time.time(),
                                            tried=results)
        _store(doc)
    return best, best_ms, results


def apply_batch(batch, device=0):
    ent = _load().get(batch_key(batch, device))
    if not ent:
        return False
    batch.set_tuning(pair_seg=ent["pair_seg"], graph_steps=ent.get("graph_steps", 50))
    return True


def apply(engine, device=0):
    """Apply the cached choice for this engine's bucket; True if one existed."""
    ent = _load().get(key_for(engine, device))
    if not ent:
        return False
    engine.set_tuning(**{k: ent[k] for k in ("force_kernel", "pair_seg", "sort_every", "source_split",
                                             "targets_per_thread") if k in ent})
    return True
