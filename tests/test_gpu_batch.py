"""Batches of independent boxes (yk_batch_*) through the C-ABI.

Each box of a batch must give what the single-box engine gives (FP64:
2-norm relative 1e-12; the batch runs pure-ion boxes through the mixture
kernels, which changes only rounding) and must give bit-identical results
whether it runs alone or among other boxes, because its work items write only
its own scratch rows and its slot order depends only on its own positions.
"""
import numpy as np
import pytest

from yukawamd_b200 import abi, configs
from yukawamd_b200.engine import Batch, Engine

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def ion_boxes():
    return [configs.pure_ion(700, 8, 16, 1.0, 175.0, seed=1),
            configs.ion_mixture(1500, [6, 8, 26], [0.2, 0.7, 0.1], 0.5, 150.0, seed=2),
            configs.pure_ion(129, 26, 52, 2.0, 60.0, seed=3),
            configs.ion_mixture(3001, [6, 8], [0.5, 0.5], 1.2, 90.0, seed=4),
            configs.pure_ion(1, 6, 12, 1.0, 100.0, seed=5)]


def nucleon_boxes():
    return [configs.nucleon(800, 0.4, 0.05, 1.0, 10.0, 2.0, seed=6),
            configs.nucleon(2000, 0.3, 0.05, 1.0, 10.0, 2.0, seed=7)]


@pytest.mark.parametrize("prec,tol", [(abi.YK_PREC_FP64, 1e-12), (abi.YK_PREC_MIXED, 1e-6)],
                         ids=["fp64", "mixed"])
@pytest.mark.parametrize("kind", ["ion", "nucleon"])
def test_batch_accel_matches_single_boxes(gpu, kind, prec, tol):
    boxes = ion_boxes() if kind == "ion" else nucleon_boxes()
    with Batch(boxes, precision=prec, mix_mode=abi.YK_MIX_FIXED) as b:
        sc = b.accel(True)
        states = [b.get_state(r) for r in range(b.nrep)]
    for r, w in enumerate(boxes):
        fixed = abi.YK_MIX_FIXED
        with Engine(w, precision=prec, mix_mode=fixed) as e:
            s = e.accel(True)
            a = e.a.copy()
        n = w.n
        ab = states[r][3]
        if n > 1:
            assert _rel(ab[:3 * n], a[:3 * n]) <= tol, (kind, r)
            assert _rel(ab[3 * n:], a[3 * n:]) <= max(tol, 1e-12), (kind, r)
            assert abs(sc[r].ev - s.ev) <= tol * abs(s.ev)
            assert abs(sc[r].px - s.px) <= tol * abs(s.px)


@pytest.mark.parametrize("prec,tol", [(abi.YK_PREC_FP64, 1e-12), (abi.YK_PREC_MIXED, 1e-6)],
                         ids=["fp64", "mixed"])
@pytest.mark.parametrize("kind", ["ion", "nucleon"])
def test_batch_accel_matches_oracle(gpu, kind, prec, tol):
    """Every box of a batch against the CPU oracle's accel
    (int_ion_pure.f:98-254, int_ion_mix.f:105-295, int_nn.f:130-345) on the
    same positions: forces and the packed sums by 2-norm, ev and px."""
    from oracle.oracle import Oracle
    orc = Oracle("double", threads=8)
    boxes = ion_boxes() if kind == "ion" else nucleon_boxes()
    with Batch(boxes, precision=prec, mix_mode=abi.YK_MIX_FIXED) as b:
        sc = b.accel(True)
        states = [b.get_state(r) for r in range(b.nrep)]
    for r, w in enumerate(boxes):
        n = w.n
        if n < 2:
            continue
        p = w.yk_params(mix_mode=abi.YK_MIX_FIXED)
        a_ref, s_ref = orc.accel(p, w.x, w.zii, w.aii, True)
        ab = states[r][3]
        assert _rel(ab[:3 * n], a_ref[:3 * n]) <= tol, (kind, r)
        assert _rel(ab[3 * n:], a_ref[3 * n:]) <= max(tol, 1e-12) * 10, (kind, r)
        assert abs(sc[r].ev - s_ref.ev) <= tol * abs(s_ref.ev), (kind, r)
        assert abs(sc[r].px - s_ref.px) <= tol * abs(s_ref.px), (kind, r)


def test_batch_steps_match_single_boxes(gpu):
    boxes = ion_boxes()[:4]
    steps, me = 60, 10
    with Batch(boxes, mix_mode=abi.YK_MIX_FIXED) as b:
        b.accel(True)
        ser, ms = b.run(steps, me)
        states = [b.get_state(r) for r in range(b.nrep)]
    assert ms > 0.0
    for r, w in enumerate(boxes):
        with Engine(w, mix_mode=abi.YK_MIX_FIXED) as e:
            e.accel(True)
            s1 = e.run(steps, me)
            x, v, _, _ = e.get_state()
        assert _rel(states[r][0], x) <= 1e-12
        assert _rel(states[r][1], v) <= 1e-9
        last = ser[(steps - 1) * b.nrep + r]
        assert abs(last.ev - s1[steps - 1].ev) <= 1e-9 * abs(s1[steps - 1].ev)
        assert abs(last.ek - s1[steps - 1].ek) <= 1e-9 * abs(s1[steps - 1].ek)
        assert last.time == s1[steps - 1].time


@pytest.mark.parametrize("prec", [abi.YK_PREC_FP64, abi.YK_PREC_MIXED], ids=["fp64", "mixed"])
def test_box_alone_equals_box_in_the_mix(gpu, prec):
    boxes = ion_boxes()
    target = 3
    steps = 73
    with Batch(boxes, precision=prec) as b:
        b.accel(True)
        ser_mix, _ = b.run(steps, 7)
        st_mix = b.get_state(target)
    with Batch([boxes[target]], precision=prec) as b1:
        b1.accel(True)
        ser_one, _ = b1.run(steps, 7)
        st_one = b1.get_state(0)
    for A, B in zip(st_mix, st_one):
        assert np.array_equal(A, B)
    for s in range(steps):
        assert bytes(ser_mix[s * len(boxes) + target]) == bytes(ser_one[s])


def test_batch_rejects_mixed_kinds(gpu):
    from yukawamd_b200._lib import EngineError
    with pytest.raises(EngineError) as ei:
        Batch([ion_boxes()[0], nucleon_boxes()[0]])
    assert ei.value.code == abi.YK_ERR_ARG


def test_sort_cadence_changes_nothing_but_speed(gpu):
    """sort_every only sets when the slot order is refreshed.  The engine's
    default is 4; a batch's tuning round-trips (0 -> the automatic 4, -1 ->
    only at the start of each graph); and 23 steps in graphs of 10 plus 3
    eager steps (where the batch counts the steps since its last sort) end
    at the same positions under every cadence, to summation-order
    rounding."""
    boxes = ion_boxes()
    with Engine(boxes[1]) as e:
        assert e.tuning().sort_every == 4
    res = {}
    for se in (0, 1, 7, -1):
        with Batch(boxes, mix_mode=abi.YK_MIX_FIXED) as b:
            t = b.set_tuning(graph_steps=10, sort_every=se)
            assert t.sort_every == {0: 4, -1: -1}.get(se, se) and t.graph_steps == 10
            b.accel(True)
            b.run(23, 5, series=False)
            res[se] = [b.get_state(r)[0] for r in range(b.nrep)]
    for se in (1, 7, -1):
        for r in range(len(boxes)):
            assert _rel(res[se][r], res[0][r]) <= 1e-12, (se, r)


def test_batch_tuning_changes_nothing_but_speed(gpu):
    """pair_seg only re-cuts the work items: accelerations agree with the
    default cut to summation-order rounding, and a graph run after the
    re-cut continues correctly."""
    from yukawamd_b200 import tune
    boxes = ion_boxes()
    with Batch(boxes, mix_mode=abi.YK_MIX_FIXED) as b:
        b.accel(True)
        a0 = [b.get_state(r)[3] for r in range(b.nrep)]
        assert b.tuning().pair_seg == 8
        t = b.set_tuning(pair_seg=3, graph_steps=20)
        assert t.pair_seg == 3 and t.graph_steps == 20
        b.accel(True)
        a1 = [b.get_state(r)[3] for r in range(b.nrep)]
        for r, w in enumerate(boxes):
            n = w.n
            if n > 1:
                assert _rel(a1[r][:3 * n], a0[r][:3 * n]) <= 1e-13
        best, best_ms, tried = tune.tune_batch(b, segs=(8, 3), steps=20, save=False)
        assert best in (8, 3) and best_ms > 0 and len(tried) == 2
        assert b.tuning().pair_seg == best
        b.run(45, 10, series=False)
