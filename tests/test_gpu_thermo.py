"""GPU parity of the driver's O(N) passes on the device state against the
oracle: ttot, tnorm, cancel_vcom (gen_utils.f:40-110) and strain
(strain.f:19-82).

Tolerances (stated here, used below):
  ttot, tnorm, cancel_vcom   relative <= 1e-13 (the sums run in a different
                             order than the oracle's loop; every other
                             operation is the reference's, correctly rounded)
  strain                     new edge lengths relative <= 1e-15 (same host
                             formula); wrapped positions bit-identical
"""
import numpy as np
import pytest

from oracle.oracle import Oracle
from yukawamd_b200 import abi, configs
from yukawamd_b200.engine import Engine

from helpers import rel, rel_norm

pytestmark = pytest.mark.gpu

TOL = 1e-13


@pytest.fixture(scope="module")
def orc():
    return Oracle("double", threads=8)


def _hot(w, seed):
    """A velocity field with centre-of-mass motion and the wrong temperature."""
    rng = np.random.default_rng(seed)
    return w.v * 1.7 + rng.normal(0.0, 1e-3, size=w.v.shape) + 3e-4


@pytest.mark.parametrize("kind", ["pure", "mix", "nn"])
def test_ttot_tnorm_cancel_vcom(gpu, orc, kind):
    w = {"pure": configs.pure_ion_ocp(81, 2000),
         "mix": configs.ion_mixture_cfg(82, 3001),
         "nn": configs.nucleon_matter(83, 2500)}[kind]
    p = w.yk_params()
    v0 = _hot(w, 7)
    with Engine(p, w.x, v0, w.zii, w.aii) as e:
        assert rel(e.ttot(), orc.ttot(p, v0, w.aii)) <= TOL
        e.tnorm()
        v_ref = v0.copy()
        orc.tnorm(p, v_ref, w.aii)
        assert rel_norm(e.get_state()[1], v_ref) <= TOL
        assert rel(e.ttot(), 1.5 * p.kT) <= TOL

        e.set_state(v=v0)
        e.cancel_vcom()
        v_ref = v0.copy()
        orc.cancel_vcom(p, v_ref, w.aii)
        v_gpu = e.get_state()[1]
        assert rel_norm(v_gpu, v_ref) <= TOL
        mom = (w.aii[:, None] * v_gpu.reshape(-1, 3)).sum(0)
        scale = (w.aii[:, None] * np.abs(v_gpu.reshape(-1, 3))).sum(0)
        assert np.all(np.abs(mom) <= 1e-12 * scale)
        assert rel(e.ttot(), 1.5 * p.kT) <= TOL


def test_cancel_vcom_then_dynamics(gpu, orc):
    """The device passes leave the engine consistent: a step after them
    matches the oracle's step after its own passes."""
    w = configs.ion_mixture_cfg(84, 1500)
    p = w.yk_params()
    v0 = _hot(w, 8)
    with Engine(p, w.x, v0, w.zii, w.aii) as e:
        e.accel(True)
        e.cancel_vcom()
        e.newton(True)
        x_gpu, v_gpu, _vo, a_gpu = e.get_state()
    a = np.zeros(3 * (w.n + 3))
    a_ref, _ = orc.accel(p, w.x, w.zii, w.aii, True)
    a[:] = a_ref
    x, v, vold = w.x.copy(), v0.copy(), np.zeros_like(v0)
    orc.cancel_vcom(p, v, w.aii)
    orc.newton(p, x, v, vold, a, w.zii, w.aii, True)
    assert rel_norm(x_gpu, x) <= 1e-12
    assert rel_norm(v_gpu, v) <= 1e-11


NO = 1000.0     # md_globals.f: no strain in that direction


@pytest.mark.parametrize("deps", [(NO, NO, NO), (2e-3, NO, NO), (NO, -3e-3, NO), (2e-3, 1e-3, NO),
                                  (NO, NO, -4e-3), (1e-3, NO, 2e-3), (NO, 1e-3, -1e-3),
                                  (1e-3, -2e-3, 3e-3)],
                         ids=["none", "x", "y", "xy", "z", "xz", "yz", "xyz"])
def test_strain_cases(gpu, orc, deps):
    w = configs.pure_ion_ocp(85, 1200)
    p = w.yk_params()
    xl0 = [t for t in p.xl]
    # push some particles just past the far faces so the wrap has work
    x0 = w.x.copy().reshape(-1, 3)
    for k in range(3):
        x0[k::7, k] = p.xl[k] * (1.0 - 1e-7)
    x0 = x0.reshape(-1)
    with Engine(p, x0, w.v, w.zii, w.aii) as e:
        for _ in range(3):
            xl_gpu = e.strain(deps, xl0)
        x_gpu = e.get_state()[0]
        s = e.accel(True)
        a_gpu = e.a.copy()
    xl = np.array(xl0, dtype=float)
    x = x0.copy()
    for _ in range(3):
        orc.strain(p, x, xl, xl0, deps)
    for k in range(3):
        assert rel(xl_gpu[k], xl[k]) <= 1e-15
    assert np.array_equal(x_gpu, x)
    p2 = w.yk_params()
    for k in range(3):
        p2.xl[k] = xl_gpu[k]
    a_ref, s_ref = orc.accel(p2, x, w.zii, w.aii, True)
    assert rel_norm(a_gpu[:3 * w.n], a_ref[:3 * w.n]) <= 1e-12
    assert rel(s.ev, s_ref.ev) <= 1e-12


def test_thermo_argument_checks(gpu):
    w = configs.pure_ion_ocp(86, 100)
    p = w.yk_params()
    p.kT = 0.0
    with Engine(p, w.x, w.v, w.zii, w.aii) as e:
        with pytest.raises(Exception):
            e.tnorm()
        with pytest.raises(Exception):
            e.cancel_vcom()
        assert e.ttot() > 0.0
        with pytest.raises(Exception):
            e.strain((-1e6, NO, NO), list(p.xl))      # would make xl(1) negative


@pytest.mark.parametrize("kind", ["pure", "mix", "nn"])
def test_vtot_matches_oracle_and_keeps_state(gpu, orc, kind):
    """yk_vtot against the oracle's restatement of vtot_* (energy per particle
    and pressure, relative <= 1e-12), leaving the state's accelerations alone."""
    w = {"pure": configs.pure_ion_ocp(87, 1500),
         "mix": configs.ion_mixture_cfg(88, 2001),
         "nn": configs.nucleon_matter(89, 1800)}[kind]
    p = w.yk_params()
    with Engine(p, w.x, w.v, w.zii, w.aii) as e:
        e.accel(False)
        a0 = e.get_state()[3]
        ev, px = e.vtot()
        a1 = e.get_state()[3]
    ev_ref, px_ref = orc.vtot(p, w.x, w.zii)
    assert rel(ev, ev_ref) <= 1e-12 and rel(px, px_ref) <= 1e-12
    assert np.array_equal(a0, a1)


@pytest.mark.parametrize("kind,n", [("pure", 2000), ("mix", 1537), ("nn", 1300)])
def test_gofr_counts_equal_oracle(gpu, orc, kind, n):
    """yk_gofr_counts bins every pair as the reference's g does (g.f:55-66):
    the counts equal the oracle's bin for bin, two calls add up, and the state
    is untouched."""
    w = {"pure": configs.pure_ion_ocp(91, n), "mix": configs.ion_mixture_cfg(92, n),
         "nn": configs.nucleon_matter(93, n)}[kind]
    p = w.yk_params()
    with Engine(p, w.x, w.v, w.zii, w.aii) as e:
        e.run(3, 0, series=False)
        x = e.get_state()[0]
        for nbin in (50, 777, 8192):
            c = e.gofr_counts(nbin)
            assert np.array_equal(c, orc.gofr_counts(p, x, nbin)), nbin
            e.gofr_counts(nbin, c)
            assert np.array_equal(c, 2 * orc.gofr_counts(p, x, nbin))
        assert np.array_equal(e.get_state()[0], x)
        with pytest.raises(Exception):
            e.gofr_counts(8193)
