"""Serving loop: admission logic (CPU) and continuous batching (GPU).

Tolerance for "the same alone and in the mix": a run's arithmetic depends only
on its own box, but the Morton order (and so the summation order) is
refreshed whenever its group is rebuilt, and rebuilds happen at different
steps alone and in a mix.  FP64 runs of a few hundred steps therefore agree to
rounding level amplified by the dynamics: positions within 1e-9 relative
(2-norm) and chunk-end energies within 1e-9 relative.
"""
import numpy as np
import pytest

from yukawamd_b200 import abi, configs
from yukawamd_b200.serve import Request, Server, admit, drift, footprint_bytes, make_requests


def test_footprint_grows_with_n():
    assert footprint_bytes(1) > 0
    small, big = footprint_bytes(1000), footprint_bytes(100000)
    assert big > 100 * small
    # half-pair scratch dominates at large n: the source-side partials take
    # n^2/128 * 12 bytes, the target-side partials another ~25 % at seg = 8
    n = 131072
    assert n ** 2 / 128 * 12 < footprint_bytes(n) < 1.4 * n ** 2 / 128 * 12


def test_admission_is_fifo_and_respects_the_budget():
    ws = [configs.pure_ion(n, 8, 16, 1.0, 175.0, seed=n) for n in (500, 4000, 800, 300)]
    reqs = [Request(i, w, 100) for i, w in enumerate(ws)]
    budget = footprint_bytes(500) + footprint_bytes(4000) + footprint_bytes(800) // 2
    got, used = admit(reqs, 0, budget)
    assert [r.rid for r in got] == [0, 1]          # 800 does not fit; 300 waits behind it
    assert used == footprint_bytes(500) + footprint_bytes(4000)
    got, used = admit(reqs, 0, 10 ** 15)
    assert [r.rid for r in got] == [0, 1, 2, 3]


def test_shadow_requests_and_drift():
    stream = configs.request_stream(seed=1, count=20, nmax=2000, smax=300)
    reqs = make_requests(stream, shadow_every=16)
    twins = [r for r in reqs if r.shadow_of >= 0]
    assert len(twins) == 2 and all(t.precision == abi.YK_PREC_FP64 for t in twins)
    assert drift([(10, 1.0), (20, 1.0 + 1e-6), (30, 1.0 - 2e-6)]) == pytest.approx(2e-6)


def _stream():
    ws = [configs.pure_ion(900, 8, 16, 1.0, 175.0, seed=31),
          configs.ion_mixture(1600, [6, 8, 26], [0.2, 0.7, 0.1], 0.5, 150.0, seed=32),
          configs.nucleon(1200, 0.4, 0.05, 1.0, 10.0, 2.0, seed=33),
          configs.pure_ion(3000, 26, 52, 1.5, 80.0, seed=34),
          configs.nucleon(700, 0.3, 0.05, 1.0, 10.0, 2.0, seed=35)]
    steps = [230, 160, 310, 120, 275]
    arrivals = [0.0, 0.05, 0.1, 0.3, 0.35]
    return [Request(i, w, s, abi.YK_PREC_FP64, t) for i, (w, s, t) in enumerate(zip(ws, steps, arrivals))]


@pytest.mark.gpu
def test_served_run_equals_run_alone(gpu):
    mix = _stream()
    srv = Server(hbm_budget=8 << 30, chunk=50)
    rep = srv.run(mix)
    assert rep["runs"] == len(mix)
    assert rep["latency_p99_s"] >= rep["latency_p50_s"] > 0.0
    assert rep["pairs_per_s"] > 0.0
    for r in mix:
        assert r.steps_done == r.steps
        alone = Request(100 + r.rid, r.workload, r.steps, abi.YK_PREC_FP64, 0.0)
        Server(hbm_budget=8 << 30, chunk=50).run([alone])
        x_rel = np.linalg.norm(r.final_x - alone.final_x) / np.linalg.norm(alone.final_x)
        assert x_rel <= 1e-9, (r.rid, x_rel)
        assert len(r.energies) >= 1
        e_mix = dict(r.energies)
        e_one = dict(alone.energies)
        common = sorted(set(e_mix) & set(e_one))
        assert common, r.rid
        for s in common:
            assert abs(e_mix[s] - e_one[s]) <= 1e-9 * abs(e_one[s])


@pytest.mark.gpu
def test_mixed_runs_with_fp64_shadow(gpu):
    stream = configs.request_stream(seed=7, count=6, rate_per_s=20.0, nmin=512, nmax=3000,
                                    smin=100, smax=300)
    reqs = make_requests(stream, shadow_every=3)
    rep = Server(hbm_budget=8 << 30, chunk=50).run(reqs)
    assert rep["runs"] == 6
    assert len(rep["fp64_shadows"]) == 2
    for sh in rep["fp64_shadows"]:
        assert sh["drift_mixed"] < 1e-3 and sh["drift_fp64"] < 1e-3
