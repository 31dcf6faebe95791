"""The CPU oracle against the 50-digit known-answer cases, plus invariants.

The reference has no tests or golden vectors and cannot be compiled here, so
these known answers (tests/golden/make_kat.py, computed independently of the
oracle's code) are what pins the oracle.
"""
import json
import os

import numpy as np
import pytest

from oracle.oracle import Oracle
from yukawamd_b200 import abi, configs

from helpers import params_from_dict, rel, rel_norm

HERE = os.path.dirname(os.path.abspath(__file__))
KAT = json.load(open(os.path.join(HERE, "golden", "kat.json")))


@pytest.fixture(scope="module")
def orc():
    return Oracle("double", threads=1)


@pytest.mark.parametrize("case", KAT["accel"], ids=lambda c: "%s-m%d" % (c["name"], c["do_meas"]))
def test_accel_known_answers(orc, case):
    p = params_from_dict(case["params"])
    n = len(case["zii"])
    a, s = orc.accel(p, np.array(case["x"]), np.array(case["zii"]), np.array(case["aii"]),
                     case["do_meas"])
    ref = np.array(case["a"])
    assert rel_norm(a[:3 * n], ref[:3 * n]) < 5e-15
    assert rel_norm(a[3 * n:], ref[3 * n:]) < 5e-15
    for key in ("ev", "px"):
        assert rel(getattr(s, key), case[key]) < 5e-15
    assert rel_norm(np.array(s.pp), np.array(case["pp"])) < 5e-15


@pytest.mark.parametrize("case", KAT["verlet"], ids=lambda c: "%s-m%d" % (c["name"], c["do_meas"]))
def test_verlet_known_answers(orc, case):
    p = params_from_dict(case["params"])
    n = len(case["zii"])
    x = np.array(case["x0"])
    v = np.array(case["v0"])
    a = np.zeros(3 * (n + 3))
    a[:3 * n] = case["a0"]
    vold = np.zeros(3 * n)
    s = orc.newton(p, x, v, vold, a, np.array(case["zii"]), np.array(case["aii"]),
                   case["do_meas"])
    L = max(case["params"]["xl"])
    assert np.allclose(x, case["x"], rtol=0.0, atol=1e-15 * L)       # ~ulp(L)
    assert rel_norm(v, np.array(case["v"])) < 1e-15
    assert np.allclose(a[:3 * n], case["a"], rtol=1e-15, atol=1e-40)
    if "vold" in case:
        assert np.array_equal(vold, np.array(case["vold"]))
    assert rel(s.ek, case["ek"]) < 1e-15
    assert rel_norm(np.array(s.pp), np.array(case["pp"])) < 1e-15
    assert s.time == p.dt


def test_rncut_matches_reference_value(orc):
    # input1.F:296-311 with the md_globals.f:127-130 defaults
    assert abs(orc.rncut() - 11.4918) < 1e-4
    assert orc.rncut() == configs.rncut_auto()


def test_thomas_fermi(orc):
    # electron density 0.05*0.4 fm^-3 -> q_TF / hbar c
    got = orc.thomas_fermi_xmuc(0.4 * 1000, 0.05, 1000)
    assert got == pytest.approx(configs.thomas_fermi_xmuc(400.0, 0.05, 1000), rel=1e-14)
    assert 0.01 < got < 0.2


def _small(w, n):
    """First n particles of a workload, box rescaled to keep the density."""
    from dataclasses import replace
    scale = (n / w.n) ** (1.0 / 3.0)
    params = dict(w.params)
    L = [t * scale for t in params["xl"]]
    params["xl"] = L
    params["rccut"] = min(params["rccut"], 0.5 * L[0] * 0.99)
    x = (w.x[:3 * n] * scale).copy()
    return replace(w, params=params, x=x, v=w.v[:3 * n].copy(), zii=w.zii[:n].copy(),
                   aii=w.aii[:n].copy())


@pytest.mark.parametrize("kind", ["pure", "mix", "nn"])
def test_newton_third_law(orc, kind):
    w = {"pure": configs.pure_ion_ocp(11, 300),
         "mix": configs.ion_mixture_cfg(12, 300),
         "nn": configs.nucleon_matter(13, 300)}[kind]
    p = w.yk_params(mix_mode=abi.YK_MIX_FIXED)
    a, _ = orc.accel(p, w.x, w.zii, w.aii, True)
    n = w.n
    F = a[:3 * n].reshape(n, 3) * (w.aii[:, None] * p.xmass)
    scale = np.abs(F).sum(0)
    assert np.all(np.abs(F.sum(0)) <= 1e-12 * scale)


def test_translation_invariance(orc):
    w = configs.pure_ion_ocp(21, 200)
    p = w.yk_params()
    a0, s0 = orc.accel(p, w.x, w.zii, w.aii, True)
    L = np.array(list(p.xl))
    x1 = (w.x.reshape(-1, 3) + np.array([0.3, 0.71, 0.05]) * L) % L
    a1, s1 = orc.accel(p, x1.reshape(-1), w.zii, w.aii, True)
    assert rel_norm(a1[:3 * w.n], a0[:3 * w.n]) < 1e-12
    assert rel(s1.ev, s0.ev) < 1e-12


def test_permutation_invariance(orc):
    w = configs.ion_mixture_cfg(22, 250)
    p = w.yk_params(mix_mode=abi.YK_MIX_FIXED)
    a0, s0 = orc.accel(p, w.x, w.zii, w.aii, True)
    perm = np.random.default_rng(0).permutation(w.n)
    x1 = w.x.reshape(-1, 3)[perm].reshape(-1)
    a1, s1 = orc.accel(p, x1, w.zii[perm], w.aii[perm], True)
    A0 = a0[:3 * w.n].reshape(-1, 3)[perm]
    assert rel_norm(a1[:3 * w.n], A0.reshape(-1)) < 1e-12
    assert rel(s1.ev, s0.ev) < 1e-12
    assert rel(s1.px, s0.px) < 1e-12


def test_mix_compat_quirk(orc):
    """compat: a(:,n-1) lacks zii(n-1) (int_ion_mix.f:158,201); fixed has it."""
    w = configs.ion_mixture_cfg(23, 120)
    pc = w.yk_params(mix_mode=abi.YK_MIX_COMPAT)
    pf = w.yk_params(mix_mode=abi.YK_MIX_FIXED)
    ac, _ = orc.accel(pc, w.x, w.zii, w.aii, False)
    af, _ = orc.accel(pf, w.x, w.zii, w.aii, False)
    n = w.n
    assert np.array_equal(ac[:3 * (n - 1)], af[:3 * (n - 1)])
    assert np.allclose(af[3 * (n - 1):3 * n], w.zii[n - 1] * ac[3 * (n - 1):3 * n], rtol=1e-15)


def test_force_is_minus_energy_gradient(orc):
    """Central finite difference of the unshifted energy vs the force."""
    w = configs.pure_ion_ocp(24, 40)
    p = w.yk_params(rccut=1e50)      # no cutoff: the energy is smooth
    n = w.n
    a, _ = orc.accel(p, w.x, w.zii, w.aii, True)
    F = a[:3 * n] * (p.ai * p.xmass)

    def energy(x):
        _, s = orc.accel(p, x, w.zii, w.aii, True)
        return s.ev * n

    h = 1e-4
    for e in (0, 7, 3 * n - 1):
        xp = w.x.copy()
        xm = w.x.copy()
        xp[e] += h
        xm[e] -= h
        g = (energy(xp) - energy(xm)) / (2 * h)
        assert F[e] == pytest.approx(-g, rel=1e-6, abs=1e-10 * np.abs(F).max())


def test_vtot_matches_accel_energy(orc):
    for w in (configs.pure_ion_ocp(25, 150), configs.nucleon_matter(26, 150)):
        p = w.yk_params()
        _, s = orc.accel(p, w.x, w.zii, w.aii, True)
        ev, pr = orc.vtot(p, w.x, w.zii)
        assert rel(ev, s.ev) < 1e-12
        assert rel(pr, s.px) < 1e-12


def test_openmp_threads_agree(orc):
    w = configs.ion_mixture_cfg(27, 400)
    p = w.yk_params()
    a1, s1 = orc.accel(p, w.x, w.zii, w.aii, True)
    o4 = Oracle("double", threads=4)
    a4, s4 = o4.accel(p, w.x, w.zii, w.aii, True)
    o4.set_threads(1)
    assert rel_norm(a4[:3 * w.n], a1[:3 * w.n]) < 1e-13
    assert rel(s4.ev, s1.ev) < 1e-13


def test_long_double_variant_agrees(orc):
    w = configs.nucleon_matter(28, 300)
    p = w.yk_params()
    a1, s1 = orc.accel(p, w.x, w.zii, w.aii, True)
    ld = Oracle("long_double")
    a2, s2 = ld.accel(p, w.x, w.zii, w.aii, True)
    assert ld.lib.orc_long_double_accum() == 1
    assert rel_norm(a1[:3 * w.n], a2[:3 * w.n]) < 1e-13
    assert rel(s1.ev, s2.ev) < 1e-13


def test_cancel_vcom_and_tnorm(orc):
    w = configs.ion_mixture_cfg(29, 500)
    p = w.yk_params()
    v = w.v.copy() + 0.01
    orc.cancel_vcom(p, v, w.aii)
    mom = (w.aii[:, None] * v.reshape(-1, 3)).sum(0)
    assert np.all(np.abs(mom) < 1e-12 * (w.aii[:, None] * np.abs(v.reshape(-1, 3))).sum(0))
    assert orc.ttot(p, v, w.aii) == pytest.approx(1.5 * p.kT, rel=1e-13)


def test_strain_volume_preserving(orc):
    w = configs.pure_ion_ocp(30, 64)
    p = w.yk_params()
    xl0 = np.array(list(p.xl))
    xl = xl0.copy()
    x = w.x.copy()
    deps = np.array([1e-4, 1000.0, 1000.0])
    for _ in range(5):
        orc.strain(p, x, xl, xl0, deps)
    assert np.prod(xl) == pytest.approx(np.prod(xl0), rel=1e-13)
    assert xl[0] > xl0[0]
    assert np.all(x.reshape(-1, 3) <= xl)
