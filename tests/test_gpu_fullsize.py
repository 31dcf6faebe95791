"""GPU parity at the benchmark sizes and at the minimum-image boundary.

Every particle of the full-size boxes is checked against one complete CPU
oracle call (OpenMP over the host cores, a few seconds each):
  * the ion mixture of int_ion_mix.f:105-295 at N = 55,296 (kappa = 0.5),
  * nucleon matter of int_nn.f:130-345 at N = 51,200 (x_p = 0.4, n_B = 0.05
    fm^-3): HPP Gaussians inside rncut plus the uncut minimum-image p-p
    screened Coulomb, where many proton pairs sit near |d| = L/2 per axis.
Tolerances (as in test_gpu_parity.py): FP64 forces 2-norm relative <= 1e-12,
ev, vir, px <= 1e-12, pp <= 1e-12; mixed forces <= 1e-6, ev, vir, px <= 1e-6,
pp <= 1e-5.  The nucleon test also checks, per axis, the 64 rows whose
proton partners come closest to |d| = L/2 (FP64 <= 1e-12 over those rows).

test_image_decisions_at_half_box builds proton pairs at |d| = L/2 + delta,
delta from 0 to 1e-3 fm, with only the Coulomb term on, so that a pair given
the wrong image flips a force term of a few per cent of its row's force: the
FP64 and mixed forms must take the reference's decision
(int_nn.f:190-195: d - L if d > L/2, d + L if d < -L/2) on every pair.
"""
import os

import numpy as np
import pytest

from oracle.oracle import Oracle
from yukawamd_b200 import abi, configs
from yukawamd_b200.engine import Engine

from helpers import rel, rel_norm

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def orc():
    return Oracle("double", threads=os.cpu_count() or 8)


def _tols(prec):
    if prec == abi.YK_PREC_FP64:
        return 1e-12, 1e-12, 1e-12
    return 1e-6, 1e-6, 1e-5


def _check(e_a, s, a_ref, s_ref, n, prec):
    ft, st, pt = _tols(prec)
    assert rel_norm(e_a[:3 * n], a_ref[:3 * n]) <= ft
    assert rel_norm(e_a[3 * n:], a_ref[3 * n:]) <= pt
    for k in ("ev", "vir", "px"):
        assert rel(getattr(s, k), getattr(s_ref, k)) <= st, k
    assert rel_norm(np.array(s.pp), np.array(s_ref.pp)) <= pt


@pytest.fixture(scope="module")
def mix_ref(orc):
    w = configs.ion_mixture_cfg(2)
    p = w.yk_params(mix_mode=abi.YK_MIX_COMPAT)
    a, s = orc.accel(p, w.x, w.zii, w.aii, True)
    return w, a, s


@pytest.fixture(scope="module")
def nuc_ref(orc):
    w = configs.nucleon_matter(3)
    a, s = orc.accel(w.yk_params(), w.x, w.zii, w.aii, True)
    return w, a, s


@pytest.mark.parametrize("tpt", [1, 2], ids=["tpt1", "tpt2"])
@pytest.mark.parametrize("prec", [abi.YK_PREC_FP64, abi.YK_PREC_MIXED], ids=["fp64", "mixed"])
def test_ion_mixture_55296_every_particle(gpu, mix_ref, prec, tpt):
    w, a_ref, s_ref = mix_ref
    with Engine(w.yk_params(precision=prec, mix_mode=abi.YK_MIX_COMPAT), w.x, w.v, w.zii, w.aii) as e:
        assert e.set_tuning(targets_per_thread=tpt).targets_per_thread == tpt
        s = e.accel(True)
        _check(e.a, s, a_ref, s_ref, w.n, prec)
        # force-only call after the measuring one: same forces within the tolerance
        e.accel(False)
        ft = _tols(prec)[0]
        assert rel_norm(e.a[:3 * w.n], a_ref[:3 * w.n]) <= ft


def _rows_nearest_half_box(w, count):
    """Per axis, the protons whose nearest proton partner along that axis is
    closest to |d| = L/2 (the minimum image's decision boundary)."""
    X = w.x.reshape(-1, 3)
    L = np.array(w.params["xl"])
    prot = np.nonzero(w.zii == 1.0)[0]
    rows = set()
    for ax in range(3):
        xs = np.sort(X[prot, ax])
        order = np.argsort(X[prot, ax])
        # for each proton, the partner coordinate closest to x + L/2 (mod L)
        tgt = np.mod(xs + L[ax] / 2, L[ax])
        pos = np.searchsorted(xs, tgt)
        gap = np.minimum(np.abs(xs[np.clip(pos, 0, len(xs) - 1)] - tgt),
                         np.abs(xs[np.clip(pos - 1, 0, len(xs) - 1)] - tgt))
        rows.update(prot[order[np.argsort(gap)[:count]]].tolist())
    return np.array(sorted(rows)), len(rows)


@pytest.mark.parametrize("prec", [abi.YK_PREC_FP64, abi.YK_PREC_MIXED], ids=["fp64", "mixed"])
def test_nucleons_51200_every_particle(gpu, nuc_ref, prec):
    _check_nucleons(nuc_ref, prec, 1)


def test_nucleons_51200_two_targets_per_thread(gpu, nuc_ref):
    _check_nucleons(nuc_ref, abi.YK_PREC_MIXED, 2)


def _check_nucleons(nuc_ref, prec, tpt):
    w, a_ref, s_ref = nuc_ref
    n = w.n
    with Engine(w.yk_params(precision=prec), w.x, w.v, w.zii, w.aii) as e:
        assert e.set_tuning(targets_per_thread=tpt).targets_per_thread == tpt
        s = e.accel(True)
        a = e.a.copy()
    _check(a, s, a_ref, s_ref, n, prec)
    rows, cnt = _rows_nearest_half_box(w, 64)
    assert cnt >= 64
    got = a[:3 * n].reshape(-1, 3)[rows]
    ref = a_ref[:3 * n].reshape(-1, 3)[rows]
    assert rel_norm(got, ref) <= _tols(prec)[0]


def _half_box_pairs(seed, n, L, deltas):
    """n protons in a cubic box of edge L; particles 2q and 2q+1 (q <
    len(deltas)) are set |d| = L/2 + deltas[q] apart along axis q % 3, in
    either direction, wrapped into [0, L)."""
    rng = np.random.default_rng(seed)
    X = rng.uniform(0.0, L, (n, 3))
    for q, dl in enumerate(deltas):
        i, j, ax = 2 * q, 2 * q + 1, q % 3
        sgn = 1.0 if q % 2 == 0 else -1.0
        X[j] = X[i] + rng.uniform(-3.0, 3.0, 3)
        X[j, ax] = X[i, ax] + sgn * (0.5 * L + dl)
    return np.ascontiguousarray(np.mod(X, L).reshape(-1))


@pytest.mark.parametrize("prec,tpt", [(abi.YK_PREC_FP64, 1), (abi.YK_PREC_MIXED, 1), (abi.YK_PREC_MIXED, 2)],
                         ids=["fp64", "mixed", "mixed-tpt2"])
def test_image_decisions_at_half_box(gpu, orc, prec, tpt):
    L, n = 30.0, 400
    base = [0.0, 1e-13, -1e-13, 1e-9, -1e-9, 1e-7, -1e-7, 1e-6, -1e-6, 1e-5, -1e-5, 1e-4, -1e-4,
            1e-3, -1e-3, 3e-3, -3e-3]
    deltas = (base * 8)[:128]
    x = _half_box_pairs(5, n, L, deltas)
    w = configs.nucleon(n, 1.0, n / L ** 3, 1.0, 10.0, 2.0, seed=6)
    p = w.yk_params(precision=prec, nuclear_on=0)
    for k in range(3):
        p.xl[k] = L
    zii = np.ones(n)
    aii = np.ones(n)
    with Engine(p, x, np.zeros(3 * n), zii, aii) as e:
        assert e.set_tuning(targets_per_thread=tpt).targets_per_thread == tpt
        e.accel(True)
        a = e.a[:3 * n].copy()
    a_ref, _ = orc.accel(p, x, zii, aii, True)
    got = a.reshape(-1, 3)[:2 * len(deltas)]
    ref = a_ref[:3 * n].reshape(-1, 3)[:2 * len(deltas)]
    tol = 1e-12 if prec == abi.YK_PREC_FP64 else 1e-5
    err = np.linalg.norm(got - ref, axis=1) / np.linalg.norm(ref, axis=1)
    assert np.all(err <= tol), (np.argmax(err), err.max())
