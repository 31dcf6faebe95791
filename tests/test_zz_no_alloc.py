"""yk_accel_noalloc: the force call that allocates no device memory.

Some callers cannot allocate device memory when they need forces: an
application whose own pool allocator owns every byte of device memory, or one
that cannot afford the device-wide synchronisation of cudaFree / cudaMalloc
on its other streams.  They pass their own device arrays to yk_accel_noalloc,
which keeps all of its working memory in one fixed array inside the library.
These tests call it through the C-ABI and check it against the ordinary entry
point, yk_accel, and against the CPU oracle, on the same positions, with the
tolerances of the parity tests: 1e-12 (2-norm, relative) for the FP64 form,
1e-6 for the mixed form.  Each case calls it twice in a row, because every
call reuses the same fixed array and must clear what it needs.

This file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from yukawamd_b200 import abi, configs
from yukawamd_b200._lib import EngineError
from yukawamd_b200.engine import Engine, accel_noalloc

pytestmark = pytest.mark.gpu

MAX_N = 4096


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def _dev(torch, arr):
    return torch.tensor(np.ascontiguousarray(arr, dtype=np.float64), device="cuda")


@pytest.fixture(scope="module")
def orc():
    from oracle.oracle import Oracle
    return Oracle("double", threads=8)


# (name, workload, overrides of its parameters, precision, tolerance, pass zii/aii)
CASES = [
    ("pure-ion OCP at the size limit", lambda: configs.pure_ion_ocp(11, MAX_N), {}, abi.YK_PREC_FP64, 1e-12, True),
    ("ion mixture", lambda: configs.ion_mixture_cfg(12, 3000), {}, abi.YK_PREC_FP64, 1e-12, True),
    ("nucleon matter", lambda: configs.nucleon_matter(13, 2000), {}, abi.YK_PREC_FP64, 1e-12, True),
    ("ion mixture, mixed precision", lambda: configs.ion_mixture_cfg(14, 2500), {}, abi.YK_PREC_MIXED, 1e-6,
     True),
    ("pure-ion OCP, mixed precision", lambda: configs.pure_ion_ocp(17, 3333), {}, abi.YK_PREC_MIXED, 1e-6, True),
    ("pure-ion OCP without zii and aii", lambda: configs.pure_ion_ocp(18, 1500), {}, abi.YK_PREC_FP64, 1e-12,
     False),
    ("B field (no pair force)", lambda: configs.pure_ion_ocp(19, 700), {"sim_type": abi.YK_SIM_BFIELD},
     abi.YK_PREC_FP64, 1e-12, True),
]


@pytest.mark.parametrize("name,make,over,prec,tol,with_z", CASES, ids=[c[0] for c in CASES])
def test_noalloc_matches_accel_twice(gpu, orc, name, make, over, prec, tol, with_z):
    import torch
    w = make()
    n = w.n
    p = w.yk_params(precision=prec, **over)
    with Engine(p, w.x, w.v, w.zii, w.aii) as e:
        s_ref = abi.YkScalars.from_buffer_copy(e.accel(True))
        a_ref = e.a.copy()
    a_orc, s_orc = orc.accel(p, w.x, w.zii, w.aii, True)
    bfield = p.sim_type == abi.YK_SIM_BFIELD
    x_d = _dev(torch, w.x)
    z_d = _dev(torch, w.zii) if with_z else None
    m_d = _dev(torch, w.aii) if with_z else None
    for call in range(2):
        a_d = torch.full((3 * (n + 3),), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        s = accel_noalloc(p, n, x_d.data_ptr(), z_d.data_ptr() if with_z else None,
                          m_d.data_ptr() if with_z else None, True, a_d.data_ptr())
        a = a_d.cpu().numpy()
        assert np.all(np.isfinite(a)), (name, call)
        if bfield:
            assert np.all(a == 0.0) and np.all(a_ref == 0.0), (name, call)
            assert s.ev == s_ref.ev and s.px == s_ref.px, (name, call)
            continue
        for ref, sr in ((a_ref, s_ref), (a_orc, s_orc)):
            assert _rel(a[:3 * n], ref[:3 * n]) <= tol, (name, call)
            assert _rel(a[3 * n:], ref[3 * n:]) <= tol, (name, call)
            for key in ("ev", "vir", "px"):
                assert abs(getattr(s, key) - getattr(sr, key)) <= tol * abs(getattr(sr, key)), (name, key)
            assert _rel(list(s.pp), list(sr.pp)) <= (tol if prec == abi.YK_PREC_FP64 else 1e-5)


def test_noalloc_rejects_sizes_beyond_its_limit(gpu):
    import torch
    n = MAX_N + 1
    w = configs.pure_ion_ocp(15, n)
    x_d = _dev(torch, w.x)
    a_d = torch.empty(3 * (n + 3), dtype=torch.float64, device="cuda")
    with pytest.raises(EngineError) as ei:
        accel_noalloc(w.yk_params(), n, x_d.data_ptr(), None, None, True, a_d.data_ptr())
    assert ei.value.code == abi.YK_ERR_ARG
    assert "at most n = 4096" in str(ei.value)


def test_noalloc_force_only_call(gpu, orc):
    import torch
    w = configs.nucleon_matter(16, 1000)
    n = w.n
    p = w.yk_params()
    with Engine(p, w.x, w.v, w.zii, w.aii) as e:
        e.accel(False)
        a_ref = e.a.copy()
    a_orc, _ = orc.accel(p, w.x, w.zii, w.aii, False)
    x_d, z_d = _dev(torch, w.x), _dev(torch, w.zii)
    a_d = torch.empty(3 * (n + 3), dtype=torch.float64, device="cuda")
    s = accel_noalloc(p, n, x_d.data_ptr(), z_d.data_ptr(), None, False, a_d.data_ptr())
    a = a_d.cpu().numpy()
    assert _rel(a[:3 * n], a_ref[:3 * n]) <= 1e-12
    assert _rel(a[:3 * n], a_orc[:3 * n]) <= 1e-12
    assert np.all(a[3 * n:] == 0.0) and s.ev == 0.0
    assert C.sizeof(s) == C.sizeof(abi.YkScalars)
