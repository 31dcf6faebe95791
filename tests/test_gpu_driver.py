"""The run driver (md.F:63-205) over the CUDA engine against the step-by-step
restatement of md.F over the oracle.

Tolerance: every record (e, p and .meas lines, group averages, the final
energies) within 1e-9 relative of the oracle run, and every time stamp and
step number equal.  The engine's FP64 forces agree with the oracle's to
~1e-14 per step; a few dozen steps of dynamics amplify that by a few orders
of magnitude at most.  The group standard deviations of statt,
sqrt(|<x^2> - <x>^2| / (n-1)), cancel <x>^2 against <x^2>, which multiplies
a relative difference d of the samples by about <x>^2 / var(x): they are
compared within 1e-5 relative.
"""
import numpy as np
import pytest

from oracle.oracle import Oracle
from yukawamd_b200 import configs
from yukawamd_b200.driver import XNOSTRAIN, RunControl, run_md
from yukawamd_b200.engine import Engine

from md_mirror import OracleEngine, md_reference

pytestmark = pytest.mark.gpu

TOL = 1e-9


def _close_rows(got, want, tols=None):
    assert len(got) == len(want)
    for g, w in zip(got, want):
        assert g[0] == w[0]
        assert g[1] == pytest.approx(w[1], rel=1e-15)
        scale = max(abs(b) for b in w[2:])      # the row's largest entry (the pp
        for c, (a, b) in enumerate(zip(g[2:], w[2:])):   # off-diagonals sit near 0)
            if tols:
                assert abs(a - b) <= tols[c] * abs(b) or abs(a - b) <= 1e-13, (g, w)
            else:
                assert abs(a - b) <= TOL * scale, (g, w)


@pytest.mark.parametrize("kind,ctl", [
    ("mix", RunControl(nwgroup=2, nwsteps=6, ngroup=3, ntot=3, nind=4, nptensor=8, ncom=5, ntnorm=6, nckpt=9)),
    ("nn", RunControl(nwgroup=1, nwsteps=4, ngroup=2, ntot=4, nind=3, nptensor=3, ncom=0, ntnorm=7)),
    ("pure", RunControl(nwgroup=1, nwsteps=3, ngroup=2, ntot=3, nind=2, nptensor=4, ntnorm=5,
                        deps=(XNOSTRAIN, 3e-3, XNOSTRAIN))),
], ids=["mix-cadence", "nn", "pure-strain"])
def test_driver_on_engine_matches_oracle_md(gpu, kind, ctl):
    w = {"mix": configs.ion_mixture_cfg(93, 900),
         "nn": configs.nucleon_matter(94, 800),
         "pure": configs.pure_ion_ocp(95, 700)}[kind]
    orc = Oracle("double", threads=8)
    ref = md_reference(OracleEngine(orc, w.yk_params(), w.x, w.v, w.zii, w.aii), ctl)
    ck = []
    with Engine(w.yk_params(), w.x, w.v, w.zii, w.aii) as e:
        res = run_md(e, ctl, on_checkpoint=lambda eng, i, t, s: ck.append((i, t)))
    assert [c[0] for c in ck] == [c[0] for c in ref["ckpt"]]
    _close_rows(res.e_lines, ref["e_lines"])
    _close_rows(res.p_lines, ref["p_lines"])
    _close_rows(res.meas, ref["meas"])
    _close_rows(res.groups, ref["groups"], tols=[TOL, 1e-5, TOL, 1e-5])    # eva dev pa dp
    for k in ("ev", "ek", "e", "px"):
        assert res.final[k] == pytest.approx(ref["final"][k], rel=TOL)
    assert np.allclose(res.final["xl"], ref["final"]["xl"], rtol=1e-15, atol=0)
