"""Serving loop: admission logic (CPU) and continuous batching (GPU).

"The same alone and in the mix": a served run lives in one slot of its
group's device-resident batch; its slot order comes from a sort of its own
particles, its work items write only its own scratch, its chunks start when
it is admitted and it stops at exactly its own step count.  So its final
positions, velocities and chunk-end energies are the same bits alone and in a
mix, in FP64 and in the mixed form; the tests state that tolerance (0) and
check it.
"""
import numpy as np
import pytest

from yukawamd_b200 import abi, configs
from yukawamd_b200.serve import Request, Server, admit, drift, footprint_bytes, make_requests, pick


def test_footprint_grows_with_n():
    assert footprint_bytes(1) > 0
    small, big = footprint_bytes(1000), footprint_bytes(100000)
    assert big > 100 * small
    # half-pair scratch dominates at large n: the source-side partials take
    # n^2/128 * 12 bytes (FP64 rows), the target-side partials up to a
    # quarter more; the mixed form's FP32 rows take half
    n = 131072
    assert n ** 2 / 128 * 12 < footprint_bytes(n) < 1.4 * n ** 2 / 128 * 12
    assert n ** 2 / 128 * 6 < footprint_bytes(n, abi.YK_PREC_MIXED) < 0.85 * n ** 2 / 128 * 12


def test_admission_passes_a_blocked_head():
    ws = [configs.pure_ion(n, 8, 16, 1.0, 175.0, seed=n) for n in (500, 4000, 800, 300)]
    reqs = [Request(i, w, 100, abi.YK_PREC_FP64) for i, w in enumerate(ws)]
    budget = footprint_bytes(500) + footprint_bytes(4000) + footprint_bytes(800) // 2
    got, used = admit(reqs, 0, budget)
    assert [r.rid for r in got] == [0, 1, 3]       # 800 does not fit; 300 passes it
    assert used == footprint_bytes(500) + footprint_bytes(4000) + footprint_bytes(300)
    got, used = admit(reqs, 0, 10 ** 15)
    assert [r.rid for r in got] == [0, 1, 2, 3]


def test_bypass_is_bounded():
    ws = [configs.pure_ion(n, 8, 16, 1.0, 175.0, seed=n) for n in (600, 200, 300)]
    reqs = [Request(i, w, 100, arrival=t) for i, (w, t) in enumerate(zip(ws, (0.0, 0.5, 1.0)))]
    fits = lambda r: r.n < 500                       # noqa: E731  (the head never fits)
    assert [r.rid for r in pick(reqs, fits, now=1.0, max_bypass_s=2.0)] == [1, 2]
    # once the head has waited max_bypass_s nothing passes it
    assert pick(reqs, fits, now=2.5, max_bypass_s=2.0) == []


def test_shadow_requests_and_drift():
    stream = configs.request_stream(seed=1, count=20, nmax=2000, smax=300)
    reqs = make_requests(stream, shadow_every=16)
    twins = [r for r in reqs if r.shadow_of >= 0]
    assert len(twins) == 2 and all(t.precision == abi.YK_PREC_FP64 for t in twins)
    assert drift([(10, 1.0), (20, 1.0 + 1e-6), (30, 1.0 - 2e-6)]) == pytest.approx(2e-6)


def _stream(prec):
    ws = [configs.pure_ion(900, 8, 16, 1.0, 175.0, seed=31),
          configs.ion_mixture(1600, [6, 8, 26], [0.2, 0.7, 0.1], 0.5, 150.0, seed=32),
          configs.nucleon(1200, 0.4, 0.05, 1.0, 10.0, 2.0, seed=33),
          configs.pure_ion(3000, 26, 52, 1.5, 80.0, seed=34),
          configs.nucleon(700, 0.3, 0.05, 1.0, 10.0, 2.0, seed=35),
          configs.pure_ion(450, 6, 12, 0.8, 120.0, seed=36)]
    steps = [230, 160, 310, 120, 275, 90]
    arrivals = [0.0, 0.05, 0.1, 0.3, 0.35, 0.4]
    return [Request(i, w, s, prec, t) for i, (w, s, t) in enumerate(zip(ws, steps, arrivals))]


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [abi.YK_PREC_FP64, abi.YK_PREC_MIXED], ids=["fp64", "mixed"])
def test_served_run_equals_run_alone(gpu, prec):
    mix = _stream(prec)
    rep = Server(hbm_budget=8 << 30, chunk=50).run(mix)
    assert rep["runs"] == len(mix)
    assert rep["latency_p99_s"] >= rep["latency_p50_s"] > 0.0
    assert rep["pairs_per_s"] > 0.0
    assert rep["pairs"] == sum(r.pairs for r in mix)
    for r in mix:
        assert r.steps_done == r.steps
        alone = Request(100 + r.rid, r.workload, r.steps, prec, 0.0)
        Server(hbm_budget=8 << 30, chunk=50).run([alone])
        assert np.array_equal(r.final_x, alone.final_x), r.rid
        assert np.array_equal(r.final_v, alone.final_v), r.rid
        assert r.energies == alone.energies, r.rid
        assert len(r.energies) == r.steps // 50


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


@pytest.mark.gpu
def test_slots_admit_run_retire(gpu):
    """A slot batch: runs enter between chunks, each takes exactly its own
    step budget inside the K-step graphs, and leaves with the state a batch
    of it alone reaches; the runs that stay are not touched."""
    from yukawamd_b200.engine import Batch, SlotBatch
    ws = [configs.pure_ion(700, 8, 16, 1.0, 175.0, seed=41),
          configs.ion_mixture(1300, [6, 8, 26], [0.2, 0.7, 0.1], 0.5, 150.0, seed=42),
          configs.pure_ion(257, 26, 52, 2.0, 60.0, seed=43)]
    steps = [70, 35, 20]
    proto = ws[0].yk_params(precision=abi.YK_PREC_FP64)
    sb = SlotBatch(proto, 4, 8000, 200)
    sb.set_tuning(graph_steps=25)
    s0, _ = sb.admit(ws[0].yk_params(mix_mode=abi.YK_MIX_FIXED), ws[0].x, ws[0].v, ws[0].zii, ws[0].aii,
                     steps[0])
    sb.run(25, 25, series=False)
    s1, _ = sb.admit(ws[1].yk_params(mix_mode=abi.YK_MIX_FIXED), ws[1].x, ws[1].v, ws[1].zii, ws[1].aii,
                     steps[1])
    s2, _ = sb.admit(ws[2].yk_params(mix_mode=abi.YK_MIX_FIXED), ws[2].x, ws[2].v, ws[2].zii, ws[2].aii,
                     steps[2])
    assert len({s0, s1, s2}) == 3
    left = sb.steps_left()
    assert left[s0] == 45 and left[s1] == 35 and left[s2] == 20
    sb.run(25, 25, series=False)
    left = sb.steps_left()
    assert left[s0] == 20 and left[s1] == 10 and left[s2] == 0
    st2 = sb.retire(s2)
    assert sb.steps_left()[s2] == -1
    sb.run(25, 25, series=False)
    left = sb.steps_left()
    assert left[s0] == 0 and left[s1] == 0
    st0, st1 = sb.retire(s0), sb.retire(s1)
    sb.close()
    # each box alone in a slot batch of its own, on the same chunks
    for w, k, st in ((ws[0], steps[0], st0), (ws[1], steps[1], st1), (ws[2], steps[2], st2)):
        one = SlotBatch(proto, 4, 8000, 200)
        one.set_tuning(graph_steps=25)
        slot, _ = one.admit(w.yk_params(mix_mode=abi.YK_MIX_FIXED), w.x, w.v, w.zii, w.aii, k)
        while one.steps_left()[slot] > 0:
            one.run(25, 25, series=False)
        ref = one.retire(slot)
        one.close()
        for A, B in zip(st, ref):
            assert np.array_equal(A, B), w.name
    # and a plain batch of the box agrees to rounding (its own sort cadence)
    with Batch([ws[1]], mix_mode=abi.YK_MIX_FIXED) as b:
        b.accel(True)
        b.run(steps[1], 0, series=False)
        x = b.get_state(0)[0]
    assert np.linalg.norm(x - st1[0]) <= 1e-12 * np.linalg.norm(x)
