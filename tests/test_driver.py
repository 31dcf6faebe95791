"""The run driver (md.F:63-205) on the CPU: its call planning, statt, the
strain edge formula, and a whole warm-up + measurement run over the oracle
that must equal the step-by-step restatement of md.F bit for bit."""
import random

import numpy as np
import pytest

from oracle.oracle import Oracle
from yukawamd_b200 import configs
from yukawamd_b200.driver import (XNOSTRAIN, RunControl, format_e_line, measures, mdmod, plan,
                                  run_md, statt, strain_edges)

from md_mirror import OracleEngine, md_reference


def test_mdmod():
    assert mdmod(7, 0) == -1 and mdmod(0, 0) == -1
    assert mdmod(6, 3) == 0 and mdmod(7, 3) == 1


def _expand(s0, calls):
    """The steps a list of yk_run calls measures (1-based global step ends)."""
    out, t = [], s0
    for k, m in calls:
        for s in range(1, k + 1):
            if m > 0 and s % m == 0:
                out.append(t + s)
        t += k
    return out, t


@pytest.mark.parametrize("nind,nptensor", [(10, 10), (10, 20), (3, 5), (0, 4), (4, 0), (0, 0), (1, 1), (7, 3)])
def test_plan_measures_exactly_the_reference_steps(nind, nptensor):
    rng = random.Random(nind * 31 + nptensor)
    for _ in range(40):
        s0 = rng.randrange(0, 50)
        s1 = s0 + rng.randrange(0, 120)
        calls = plan(s0, s1, nind, nptensor)
        got, end = _expand(s0, calls)
        assert end == s1
        want = [i + 1 for i in range(s0, s1) if measures(i + 1, nind, nptensor)]
        assert got == want
        assert all(k > 0 for k, _ in calls)


def test_plan_is_one_call_for_aligned_cadence():
    assert plan(0, 1000, 10, 10) == [(1000, 10)]
    assert plan(0, 1005, 10, 20) == [(1005, 10)]
    assert plan(0, 100, 0, 0) == [(100, 0)]
    assert len(plan(5, 1000, 10, 10)) == 2


def test_statt_matches_formula():
    xa, xa2, dx, xave, x2ave = statt(10.0, 30.0, 4, 1.0, 2.0)
    assert xa == 2.5 and xa2 == 7.5
    assert dx == pytest.approx(np.sqrt(abs(7.5 - 6.25) / 3.0))
    assert xave == 3.5 and x2ave == 2.0 + 6.25
    assert statt(5.0, 25.0, 1, 0.0, 0.0)[2] == 0.0


@pytest.mark.parametrize("sel", range(8))
def test_strain_edges_match_oracle(sel):
    orc = Oracle("double")
    w = configs.pure_ion_ocp(91, 64)
    p = w.yk_params()
    rates = (1e-3, -2e-3, 3e-3)
    deps = tuple(rates[k] if sel >> k & 1 else XNOSTRAIN for k in range(3))
    xl0 = list(p.xl)
    xl = np.array(xl0)
    mine = list(xl0)
    x = w.x.copy()
    for _ in range(4):
        orc.strain(p, x, xl, np.array(xl0), np.array(deps))
        mine = strain_edges(mine, xl0, deps, p.dt)
        assert mine == list(xl)


def test_format_e_line():
    line = format_e_line("e", 120, 1234.5, [1.0, -2.5e-3, 3.0, 4.0])
    assert line == "e     120        1234.50   1.000000000E+00  -2.500000000E-03   3.000000000E+00   4.000000000E+00"


CONTROLS = {
    "cadence": RunControl(nwgroup=2, nwsteps=5, ngroup=3, ntot=3, nind=3, nptensor=6, ncom=5,
                          ntnorm=4, nckpt=7),
    "strain": RunControl(nwgroup=1, nwsteps=3, ngroup=2, ntot=2, nind=2, nptensor=4, ncom=0,
                         ntnorm=3, deps=(4e-3, XNOSTRAIN, XNOSTRAIN)),
    "plain": RunControl(ngroup=2, ntot=4, nind=2, nptensor=0),
}


@pytest.mark.parametrize("name", list(CONTROLS))
def test_driver_equals_stepwise_md_on_the_oracle(name):
    orc = Oracle("double", threads=1)      # one thread: a fixed summation order
    w = configs.ion_mixture_cfg(92, 300)
    ctl = CONTROLS[name]
    ref_eng = OracleEngine(orc, w.yk_params(), w.x, w.v, w.zii, w.aii)
    ref = md_reference(ref_eng, ctl)

    eng = OracleEngine(orc, w.yk_params(), w.x, w.v, w.zii, w.aii)
    ck = []
    res = run_md(eng, ctl, on_checkpoint=lambda e, i, t, s: ck.append((i, t)))
    assert res.initial == ref["initial"]
    assert res.warmup == ref["warmup"]
    assert res.e_lines == ref["e_lines"]
    assert res.p_lines == ref["p_lines"]
    assert res.meas == ref["meas"]
    assert res.groups == ref["groups"]
    assert ck == ref["ckpt"]
    assert (res.evave, res.devave, res.pave, res.dpave) == (ref["evave"], ref["devave"], ref["pave"], ref["dpave"])
    for k in ("ev", "ek", "e", "px", "xl"):
        assert res.final[k] == ref["final"][k]
    assert np.array_equal(eng.x, ref_eng.x) and np.array_equal(eng.v, ref_eng.v)
    if not ctl.strained:
        assert res.calls < ctl.nwgroup * ctl.nwsteps + ctl.ngroup * ctl.ntot * ctl.nind
