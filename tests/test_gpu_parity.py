"""GPU parity: the CUDA engine through the C-ABI against the CPU oracle.

Tolerances (stated here, used below):
  FP64 form   forces  ||a_gpu - a_ref||_2 / ||a_ref||_2 <= 1e-12
              ev, vir, px relative <= 1e-12; pp and the packed raw sums
              a(:,n..n+2) by 2-norm <= 1e-12
              Verlet positions / velocities: bit-identical given identical
              accelerations ('B-field' force case)
  mixed form  forces 2-norm relative <= 1e-6; ev, px relative <= 1e-6;
              pp 2-norm relative <= 1e-5
"""
import numpy as np
import pytest

from oracle.oracle import Oracle
from yukawamd_b200 import abi, configs
from yukawamd_b200.engine import Engine, kernel_launch_count

from helpers import params_from_dict, rel, rel_norm
from rows import row_accels

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
MIX_F_TOL = 1e-6
MIX_S_TOL = 1e-6


@pytest.fixture(scope="module")
def orc():
    return Oracle("double", threads=8)


def workload(kind, n, seed):
    if kind == "pure":
        return configs.pure_ion_ocp(seed, n)
    if kind == "mix":
        return configs.ion_mixture_cfg(seed, n)
    return configs.nucleon_matter(seed, n)


def check_accel(orc, w, prec, meas, mix_mode=abi.YK_MIX_COMPAT, tuning=None):
    p = w.yk_params(precision=prec, mix_mode=mix_mode)
    n = w.n
    with Engine(p, w.x, w.v, w.zii, w.aii) as e:
        if tuning:
            e.set_tuning(**tuning)
        s = e.accel(meas)
        a_gpu = e.a.copy()
    a_ref, s_ref = orc.accel(p, w.x, w.zii, w.aii, meas)
    if prec == abi.YK_PREC_FP64:
        ft, st, pt = FP64_TOL, FP64_TOL, FP64_TOL
    else:
        ft, st, pt = MIX_F_TOL, MIX_S_TOL, 1e-5
    assert rel_norm(a_gpu[:3 * n], a_ref[:3 * n]) <= ft
    if meas:
        assert rel_norm(a_gpu[3 * n:], a_ref[3 * n:]) <= pt
        assert rel(s.ev, s_ref.ev) <= st
        assert rel(s.vir, s_ref.vir) <= st
        assert rel(s.px, s_ref.px) <= st
        assert rel_norm(np.array(s.pp), np.array(s_ref.pp)) <= pt
    else:
        assert np.all(a_gpu[3 * n:] == 0.0)
        assert s.ev == 0.0 and s.px == 0.0 and all(t == 0.0 for t in s.pp)


KERNELS = {"rows": dict(force_kernel=abi.KERNEL_ROWS),
           "pairs": dict(force_kernel=abi.KERNEL_PAIRS),
           "pairs-unsorted-seg3": dict(force_kernel=abi.KERNEL_PAIRS, sort_every=-1, pair_seg=3),
           "near": dict(force_kernel=abi.KERNEL_NEAR),
           "near-unsorted-seg3": dict(force_kernel=abi.KERNEL_NEAR, sort_every=-1, pair_seg=3),
           "pairs-split2": dict(force_kernel=abi.KERNEL_PAIRS, source_split=2),
           "pairs-split4-unsorted": dict(force_kernel=abi.KERNEL_PAIRS, sort_every=-1, source_split=4),
           "pairs-tpt2": dict(force_kernel=abi.KERNEL_PAIRS, targets_per_thread=2)}


@pytest.mark.parametrize("kern", [k for k in KERNELS if "tpt2" not in k])
@pytest.mark.parametrize("prec", [abi.YK_PREC_FP64, abi.YK_PREC_MIXED], ids=["fp64", "mixed"])
@pytest.mark.parametrize("meas", [True, False], ids=["meas", "force"])
@pytest.mark.parametrize("kind,n", [("pure", 4096), ("mix", 3000), ("nn", 3000)])
def test_accel_matches_oracle(gpu, orc, kind, n, meas, prec, kern):
    check_accel(orc, workload(kind, n, 100 + n), prec, meas, tuning=KERNELS[kern])


@pytest.mark.parametrize("kern", ["rows", "pairs", "near", "pairs-split4-unsorted"])
@pytest.mark.parametrize("n", [1, 2, 3, 17, 127, 128, 129, 255, 257])
@pytest.mark.parametrize("kind", ["pure", "mix", "nn"])
def test_ragged_sizes(gpu, orc, kind, n, kern):
    w = workload(kind, n, 7 + n)
    check_accel(orc, w, abi.YK_PREC_FP64, True, tuning=KERNELS[kern])
    check_accel(orc, w, abi.YK_PREC_FP64, False, tuning=KERNELS[kern])


@pytest.mark.parametrize("n", [2, 17, 129, 257, 513, 1500, 4000])
@pytest.mark.parametrize("sort", ["sorted", "unsorted"])
def test_mixed_nucleons_species_modes(gpu, orc, n, sort):
    """The mixed nucleon kernel's species modes (neutron warps without the
    Coulomb term and flag test where the nuclear range is short of L/2;
    proton warps on proton tiles without species tests; anything else the
    general path): species-major slot order makes single-species warps and
    tiles, the identity order mixed ones; small boxes have the nuclear range
    beyond L/2.  Measuring and force-only calls against the oracle."""
    w = workload("nn", n, 60 + n)
    tun = dict(force_kernel=abi.KERNEL_PAIRS, sort_every=50 if sort == "sorted" else -1)
    check_accel(orc, w, abi.YK_PREC_MIXED, True, tuning=tun)
    check_accel(orc, w, abi.YK_PREC_MIXED, False, tuning=tun)


@pytest.mark.parametrize("kern", ["rows", "pairs", "near"])
@pytest.mark.parametrize("mode", [abi.YK_MIX_COMPAT, abi.YK_MIX_FIXED], ids=["compat", "fixed"])
def test_mix_last_particle_mode(gpu, orc, mode, kern):
    check_accel(orc, workload("mix", 513, 5), abi.YK_PREC_FP64, False, mix_mode=mode,
                tuning=KERNELS[kern])


def test_known_answers_through_capi(gpu):
    import json
    import os
    doc = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "kat.json")))
    for case in doc["accel"]:
        p = params_from_dict(case["params"])
        n = len(case["zii"])
        with Engine(p, np.array(case["x"]), None, np.array(case["zii"]),
                    np.array(case["aii"])) as e:
            s = e.accel(case["do_meas"])
            a = e.a.copy()
        ref = np.array(case["a"])
        assert rel_norm(a[:3 * n], ref[:3 * n]) <= 1e-14, case["name"]
        if case["do_meas"]:
            assert rel_norm(a[3 * n:], ref[3 * n:]) <= 1e-14, case["name"]
            assert rel(s.ev, case["ev"]) <= 1e-14
            assert rel(s.px, case["px"]) <= 1e-14


@pytest.mark.parametrize("integ", [1, 2, 3])
@pytest.mark.parametrize("bfield", [0.0, 2.0e17], ids=["b0", "b1"])
def test_verlet_bit_exact(gpu, orc, integ, bfield):
    """'B-field' force case (a = 0): every step's x, v, vold, a must be
    bit-identical to the oracle's reference-order arithmetic."""
    w = configs.ion_mixture_cfg(31, 1000)
    p = w.yk_params(sim_type=abi.YK_SIM_BFIELD, integrator=integ, bfield=bfield)
    n = w.n
    rng = np.random.default_rng(3)
    a0 = rng.standard_normal(3 * n) * 1e-4
    x, v = w.x.copy(), w.v.copy()
    vold = np.zeros(3 * n)
    a = np.zeros(3 * (n + 3))
    a[:3 * n] = a0
    s_ref = abi.YkScalars()
    with Engine(p, w.x, w.v, w.zii, w.aii) as e:
        e.set_state(a=a0)
        for step in range(4):
            meas = step % 2 == 1
            s = e.newton(meas)
            orc.newton(p, x, v, vold, a, w.zii, w.aii, meas, s_ref)
            gx, gv, gvold, ga = e.get_state()
            assert np.array_equal(gx, x)
            assert np.array_equal(gv, v)
            assert np.array_equal(ga, a[:3 * n])
            if integ == 2:
                assert np.array_equal(gvold, vold)
            assert rel(s.ek, s_ref.ek) <= 1e-13
            assert rel_norm(np.array(s.pp), np.array(s_ref.pp)) <= 1e-13
            assert s.time == s_ref.time


@pytest.mark.parametrize("kind", ["pure", "mix", "nn"])
def test_newton_steps_match_oracle(gpu, orc, kind):
    w = workload(kind, 1500, 41)
    p = w.yk_params()
    n = w.n
    x, v = w.x.copy(), w.v.copy()
    vold = np.zeros(3 * n)
    a, s_ref = orc.accel(p, x, w.zii, w.aii, True)
    with Engine(p, w.x, w.v, w.zii, w.aii) as e:
        e.accel(True)
        for step in range(5):
            meas = step >= 3
            s = e.newton(meas)
            orc.newton(p, x, v, vold, a, w.zii, w.aii, meas, s_ref)
        gx, gv, _, ga = e.get_state()
    assert rel_norm(gx, x) <= 1e-14
    assert rel_norm(gv, v) <= 1e-12
    assert rel_norm(ga, a[:3 * n]) <= 1e-11
    assert rel(s.ev, s_ref.ev) <= 1e-11
    assert rel(s.ek, s_ref.ek) <= 1e-11
    assert rel(s.px, s_ref.px) <= 1e-11


@pytest.mark.parametrize("kern", ["rows", "pairs", "near", "pairs-tpt2"])
@pytest.mark.parametrize("prec", [abi.YK_PREC_FP64, abi.YK_PREC_MIXED], ids=["fp64", "mixed"])
def test_run_graph_equals_newton_loop(gpu, prec, kern):
    """yk_run (CUDA graphs, Morton re-sorts inside) is bit-identical to the
    same steps via yk_newton."""
    w = configs.pure_ion_ocp(51, 2000)
    p = w.yk_params(precision=prec)
    steps, me = 157, 5
    with Engine(p, w.x, w.v, w.zii, w.aii) as e1:
        e1.set_tuning(**KERNELS[kern])
        e1.accel(True)
        # global step g (1-based) measures when g > 3 and (g - 3) % me == 0,
        # which is the pattern of the two yk_run calls below
        ser1 = [abi.YkScalars.from_buffer_copy(e1.newton(g > 3 and (g - 3) % me == 0))
                for g in range(1, steps + 1)]
        st1 = e1.get_state()
    with Engine(p, w.x, w.v, w.zii, w.aii) as e2:
        e2.set_tuning(**KERNELS[kern])
        e2.accel(True)
        e2.run(3, me, series=False)          # start unaligned with the sort cadence
        ser2 = e2.run(steps - 3, me)
        st2 = e2.get_state()
    for A, B in zip(st1, st2):
        assert np.array_equal(A, B)
    assert len(ser2) == steps - 3
    for s1, s2 in zip(ser1[3:], ser2):
        assert bytes(s1) == bytes(s2)


def test_full_size_rows_and_third_law(gpu):
    """N = 55,296 ion mixture (the benchmark size): sampled rows against a
    numpy restatement, Newton's third law on the FP64 forces, and the mixed
    form against FP64."""
    w = configs.ion_mixture_cfg(2)
    n = w.n
    p = w.yk_params(mix_mode=abi.YK_MIX_FIXED)
    with Engine(p, w.x, w.v, w.zii, w.aii) as e:
        e.accel(True)
        a64 = e.a[:3 * n].copy()
    rows = np.random.default_rng(1).choice(n, 48, replace=False)
    ref = row_accels(p, w.x, w.zii, w.aii, rows)
    got = a64.reshape(-1, 3)[rows]
    assert rel_norm(got, ref) <= FP64_TOL
    F = a64.reshape(-1, 3) * (w.aii[:, None] * p.xmass)
    assert np.all(np.abs(F.sum(0)) <= 1e-11 * np.abs(F).sum(0))
    with Engine(p, w.x, w.v, w.zii, w.aii, precision=abi.YK_PREC_MIXED) as e:
        e.accel(True)
        am = e.a[:3 * n].copy()
    assert rel_norm(am, a64) <= MIX_F_TOL


def test_state_round_trip_and_box(gpu, orc):
    w = configs.pure_ion_ocp(61, 700)
    p = w.yk_params()
    with Engine(p, w.x, w.v, w.zii, w.aii) as e:
        x, v, vold, a = e.get_state()
        assert np.array_equal(x, w.x) and np.array_equal(v, w.v)
        L2 = [t * 1.01 for t in p.xl]
        e.set_box(L2)
        x2 = w.x * 1.01
        e.set_state(x=x2)
        s = e.accel(True)
        p2 = w.yk_params()
        for k in range(3):
            p2.xl[k] = L2[k]
        a_ref, s_ref = orc.accel(p2, x2, w.zii, w.aii, True)
        assert rel_norm(e.a[:3 * w.n], a_ref[:3 * w.n]) <= FP64_TOL
        assert rel(s.ev, s_ref.ev) <= FP64_TOL


def _short_cutoff(w, frac):
    """The workload with r_c = frac * L (below L/2, so that the screen's
    image integers are exact and the two-target kernel applies)."""
    import copy
    w2 = copy.deepcopy(w)
    w2.params["rccut"] = frac * min(w.params["xl"])
    return w2


TPT2 = {"tpt2": dict(force_kernel=abi.KERNEL_PAIRS, targets_per_thread=2),
        "tpt2-unsorted-seg3": dict(force_kernel=abi.KERNEL_PAIRS, sort_every=-1, pair_seg=3, targets_per_thread=2),
        "tpt2-seg1": dict(force_kernel=abi.KERNEL_PAIRS, pair_seg=1, targets_per_thread=2)}


def check_tpt2(orc, w, prec, meas, kern, mix_mode=abi.YK_MIX_COMPAT):
    """check_accel on the two-target kernel, asserting that it ran."""
    p = w.yk_params(precision=prec, mix_mode=mix_mode)
    with Engine(p, w.x, w.v, w.zii, w.aii) as e:
        assert e.set_tuning(**TPT2[kern]).targets_per_thread == 2
    check_accel(orc, w, prec, meas, mix_mode=mix_mode, tuning=TPT2[kern])


@pytest.mark.parametrize("kern", list(TPT2))
@pytest.mark.parametrize("prec", [abi.YK_PREC_FP64, abi.YK_PREC_MIXED], ids=["fp64", "mixed"])
@pytest.mark.parametrize("meas", [True, False], ids=["meas", "force"])
@pytest.mark.parametrize("kind,n", [("pure", 4096), ("mix", 3000), ("mix", 6001)])
def test_two_targets_per_thread_matches_oracle(gpu, orc, kind, n, meas, prec, kern):
    """The two-target kernel (blocks of 256 targets) against the oracle: odd
    and even tile counts, jobs cut to one and three tiles, unsorted slots."""
    check_tpt2(orc, _short_cutoff(workload(kind, n, 300 + n), 0.4), prec, meas, kern)


@pytest.mark.parametrize("n", [1, 2, 3, 17, 127, 128, 129, 255, 256, 257, 383, 385, 513])
@pytest.mark.parametrize("kind", ["pure", "mix"])
def test_two_targets_per_thread_ragged(gpu, orc, kind, n):
    """Ragged sizes, including a last block pair with one block (odd tile
    count) and partial tiles, FP64 and mixed, measuring and force-only."""
    w = _short_cutoff(workload(kind, n, 11 + n), 0.35)
    for prec in (abi.YK_PREC_FP64, abi.YK_PREC_MIXED):
        check_tpt2(orc, w, prec, True, "tpt2")
        check_tpt2(orc, w, prec, False, "tpt2-seg1")


@pytest.mark.parametrize("kern", list(TPT2))
@pytest.mark.parametrize("meas", [True, False], ids=["meas", "force"])
@pytest.mark.parametrize("n", [3000, 6001])
def test_two_targets_per_thread_nucleons(gpu, orc, n, meas, kern):
    """Nucleons, mixed form (the hi/lo displacement with the flagged exact
    image near L/2): the two-target kernel against the oracle."""
    check_tpt2(orc, workload("nn", n, 500 + n), abi.YK_PREC_MIXED, meas, kern)


@pytest.mark.parametrize("n", [1, 2, 17, 128, 129, 255, 257, 383, 385])
def test_two_targets_per_thread_nucleons_ragged(gpu, orc, n):
    w = workload("nn", n, 31 + n)
    check_tpt2(orc, w, abi.YK_PREC_MIXED, True, "tpt2")
    check_tpt2(orc, w, abi.YK_PREC_MIXED, False, "tpt2-seg1")


@pytest.mark.parametrize("mode", [abi.YK_MIX_COMPAT, abi.YK_MIX_FIXED], ids=["compat", "fixed"])
def test_two_targets_per_thread_mix_modes(gpu, orc, mode):
    w = _short_cutoff(workload("mix", 513, 5), 0.4)
    check_tpt2(orc, w, abi.YK_PREC_FP64, True, "tpt2", mix_mode=mode)


@pytest.mark.parametrize("prec", [abi.YK_PREC_FP64, abi.YK_PREC_MIXED], ids=["fp64", "mixed"])
def test_two_targets_per_thread_follows_the_box(gpu, orc, prec):
    """targets_per_thread = 2 runs on ion boxes whose screen images are exact;
    a box change that breaks that condition (the cutoff beyond L/2) takes the
    one-target kernel, and a change back returns to two; the forces match the
    oracle throughout.  Nucleon boxes report 2 in the mixed form only."""
    w = _short_cutoff(configs.ion_mixture_cfg(81, 3000), 0.4)
    p = w.yk_params(precision=prec)
    L = list(p.xl)
    with Engine(p, w.x, w.v, w.zii, w.aii) as e:
        assert e.set_tuning(force_kernel=abi.KERNEL_PAIRS, targets_per_thread=2).targets_per_thread == 2
        for scale, tpt in ((1.0, 2), (0.7, 1), (1.0, 2)):
            xl = [t * scale for t in L]
            e.set_box(xl)
            x = w.x * scale
            e.set_state(x=x)
            s = e.accel(True)
            assert e.tuning().targets_per_thread == tpt, scale
            p2 = w.yk_params(precision=prec)
            for k in range(3):
                p2.xl[k] = xl[k]
            a_ref, s_ref = orc.accel(p2, x, w.zii, w.aii, True)
            tol = FP64_TOL if prec == abi.YK_PREC_FP64 else MIX_F_TOL
            assert rel_norm(e.a[:3 * w.n], a_ref[:3 * w.n]) <= tol
            assert rel(s.ev, s_ref.ev) <= (FP64_TOL if prec == abi.YK_PREC_FP64 else MIX_S_TOL)
    wn = configs.nucleon_matter(82, 2000)
    with Engine(wn.yk_params(precision=prec), wn.x, wn.v, wn.zii, wn.aii) as e:
        # nucleons: two targets in the mixed form only
        want = 2 if prec == abi.YK_PREC_MIXED else 1
        assert e.set_tuning(force_kernel=abi.KERNEL_PAIRS, targets_per_thread=2).targets_per_thread == want


@pytest.mark.parametrize("tpt", [1, 2], ids=["tpt1", "tpt2"])
@pytest.mark.parametrize("kind", ["pure", "mix"])
def test_mixed_displacement_large_box(gpu, orc, kind, tpt):
    """The mixed form's FP32 ion displacement (hi parts on the 2^-9 fm grid,
    exact differences, a lo correction) in a box of L = 16,000 fm, just inside
    the limit for it (every coordinate below 16,384 fm), with particles
    crowded against both faces so that the hi parts are as large as they get
    and many pairs cross the periodic boundary: forces within 1e-6 RMS and
    ev, px within 1e-6 of the FP64 oracle; the FP64 form within 1e-12."""
    import copy
    w = copy.deepcopy(workload(kind, 3000, 900 + tpt))
    L = 16000.0
    rng = np.random.default_rng(77)
    X = rng.random((w.n, 3))
    # half the particles within 500 fm of a face (either side)
    edge = rng.random(w.n) < 0.5
    X[edge] = np.where(rng.random((edge.sum(), 3)) < 0.5, X[edge] * (500.0 / L), 1.0 - X[edge] * (500.0 / L))
    w.x = np.ascontiguousarray((X * L).reshape(-1))
    w.params["xl"] = [L, L, L]
    w.params["rccut"] = 0.35 * L
    w.params["xmuc"] = 1.0 / 1500.0
    for prec in (abi.YK_PREC_FP64, abi.YK_PREC_MIXED):
        p = w.yk_params(precision=prec)
        with Engine(p, w.x, w.v, w.zii, w.aii) as e:
            t = e.set_tuning(force_kernel=abi.KERNEL_PAIRS, targets_per_thread=tpt)
            assert t.targets_per_thread == tpt
        check_accel(orc, w, prec, True, tuning=dict(force_kernel=abi.KERNEL_PAIRS, targets_per_thread=tpt))


def test_kernels_actually_launch(gpu):
    w = configs.pure_ion_ocp(71, 300)
    before = kernel_launch_count()
    with Engine(w) as e:
        e.accel(True)
        e.newton(False)
        e.run(10, 0, series=False)
    assert kernel_launch_count() - before >= 2 + 4 + 40


def test_nonfinite_state_rejected(gpu):
    w = configs.pure_ion_ocp(72, 100)
    with Engine(w) as e:
        bad = w.x.copy()
        bad[5] = np.nan
        with pytest.raises(Exception) as ei:
            e.set_state(x=bad)
        assert ei.value.code == abi.YK_ERR_NONFINITE


def _reshaped(w, stretch, rccut=None):
    """The workload in a rectangular box (edges scaled by `stretch`, positions
    with them) and optionally another cutoff."""
    import copy
    w2 = copy.deepcopy(w)
    x = w2.x.reshape(-1, 3) * np.asarray(stretch)
    w2.x = np.ascontiguousarray(x.reshape(-1))
    w2.params["xl"] = [w.params["xl"][k] * stretch[k] for k in range(3)]
    if rccut is not None:
        w2.params["rccut"] = rccut
    return w2


@pytest.mark.parametrize("kern", ["rows", "pairs", "near", "pairs-tpt2"])
@pytest.mark.parametrize("prec", [abi.YK_PREC_FP64, abi.YK_PREC_MIXED], ids=["fp64", "mixed"])
@pytest.mark.parametrize("case", ["rectangular", "cutoff-at-half-box", "no-cutoff"])
def test_box_shapes_and_cutoffs(gpu, orc, case, prec, kern):
    """Rectangular boxes (edges 2 : 1 : 0.7) and cutoffs at or beyond L/2, where
    pairs straddle the minimum-image boundary: the per-pair screen's image
    integers are then not used (the exact comparisons run), and the bounding-box
    and near-list classifications meet ambiguous sources."""
    w = configs.ion_mixture_cfg(101, 2500)
    L = w.params["xl"][0]
    if case == "rectangular":
        w = _reshaped(w, (2.0, 1.0, 0.7))
    elif case == "cutoff-at-half-box":
        w = _reshaped(w, (1.0, 1.0, 1.0), rccut=0.5 * L)
    else:
        w = _reshaped(w, (1.3, 1.0, 0.8), rccut=1e50)
    check_accel(orc, w, prec, True, mix_mode=abi.YK_MIX_FIXED, tuning=KERNELS[kern])


@pytest.mark.parametrize("integ,bfield", [(1, 0.0), (3, 0.0), (2, 2.0e17), (3, 2.0e17)],
                         ids=["vv1", "vv3", "vv2-b", "vv3-b"])
def test_run_graph_equals_newton_loop_integrators(gpu, integ, bfield):
    """yk_run's CUDA graphs for the other integrators and the B field give the
    same bits as the same steps through yk_newton."""
    w = configs.ion_mixture_cfg(52, 1200)
    p = w.yk_params(integrator=integ, bfield=bfield)
    steps, me = 60, 7
    with Engine(p, w.x, w.v, w.zii, w.aii) as e1:
        e1.accel(True)
        ser1 = [abi.YkScalars.from_buffer_copy(e1.newton(g % me == 0)) for g in range(1, steps + 1)]
        st1 = e1.get_state()
    with Engine(p, w.x, w.v, w.zii, w.aii) as e2:
        e2.set_tuning(graph_steps=20)
        e2.accel(True)
        ser2 = e2.run(steps, me)
        st2 = e2.get_state()
    for A, B in zip(st1, st2):
        assert np.array_equal(A, B)
    for s1, s2 in zip(ser1, ser2):
        assert bytes(s1) == bytes(s2)
