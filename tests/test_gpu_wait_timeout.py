"""Failure path of the device-side waits, without a GPU fault.

Every wait of the force kernels on a tile copy is bounded; a wait that runs
out sets ERR_TIMEOUT in the context's error word, the kernel returns, and the
host reports YK_ERR_TIMEOUT (the engine's replacement for the reference's
md_exit, md_utils.f:158-183).  yk_wait_selftest makes both wait forms run out
on a barrier that no copy ever completes, with a short poll limit, so nothing
hangs or faults.  The test checks the status through the C-ABI and that the
same context then still computes forces equal to the oracle's.
"""
import ctypes as C

import numpy as np
import pytest

from yukawamd_b200 import abi, configs
from yukawamd_b200.engine import Engine

pytestmark = pytest.mark.gpu


def test_bounded_wait_times_out_and_context_survives(gpu):
    from oracle.oracle import Oracle
    w = configs.pure_ion_ocp(21, 600)
    p = w.yk_params()
    with Engine(p, w.x, w.v, w.zii, w.aii) as e:
        lib = e._lib
        for spins in (1, 4096):
            gave_up = C.c_int(-1)
            rc = lib.yk_wait_selftest(e._ctx, spins, C.byref(gave_up))
            assert rc == abi.YK_ERR_TIMEOUT, rc
            assert gave_up.value == 128
            msg = lib.yk_last_error(e._ctx).decode()
            assert "timed out" in msg, msg
        # out-of-range limits are argument errors, not launches
        assert lib.yk_wait_selftest(e._ctx, 0, None) == abi.YK_ERR_ARG
        assert lib.yk_wait_selftest(e._ctx, (1 << 22) + 1, None) == abi.YK_ERR_ARG
        # the error word was cleared: the next force call succeeds and is right
        e.accel(True)
        a = e.a.copy()
    a_ref, _ = Oracle("double", threads=4).accel(p, w.x, w.zii, w.aii, True)
    n = w.n
    err = np.linalg.norm(a[:3 * n] - a_ref[:3 * n]) / np.linalg.norm(a_ref[:3 * n])
    assert err <= 1e-12
