"""Asynchronous snapshots (yk_snapshot_begin / yk_snapshot_wait) and the
checkpoint writer on the device state: a snapshot holds the state at the
moment it was taken even while later steps run, and the driver's checkpoint
files hold exactly the engine's state at those steps (bit for bit)."""
import numpy as np
import pytest

from yukawamd_b200 import configs
from yukawamd_b200.driver import RunControl, run_md
from yukawamd_b200.engine import Engine, host_register, host_unregister
from yukawamd_b200.xvb import Checkpointer, read_xvb

pytestmark = pytest.mark.gpu


def test_snapshot_is_taken_before_later_steps(gpu):
    w = configs.ion_mixture_cfg(96, 5000)
    with Engine(w) as e:
        e.run(7, 0, series=False)
        x0, v0, _vo, a0 = e.get_state()
        xs, vs, as_ = (np.full(3 * w.n, np.nan) for _ in range(3))
        for b in (xs, vs, as_):
            host_register(b)
        try:
            e.snapshot_begin(xs, vs, as_)
            e.run(20, 0, series=False)               # overwrites x, v, a on the device
            e.snapshot_wait()
            x1 = e.get_state()[0]
        finally:
            for b in (xs, vs, as_):
                host_unregister(b)
    assert np.array_equal(xs, x0) and np.array_equal(vs, v0) and np.array_equal(as_, a0)
    assert not np.array_equal(x1, x0)


def test_snapshot_unregistered_buffers_and_partial(gpu):
    w = configs.pure_ion_ocp(97, 900)
    with Engine(w) as e:
        e.run(3, 0, series=False)
        x0, v0, _vo, _a = e.get_state()
        v = np.empty(3 * w.n)
        e.snapshot_begin(None, v, None)
        e.snapshot_begin(None, v, None)               # waits for the first one
        e.snapshot_wait()
        e.snapshot_wait()                             # nothing in flight: returns
    assert np.array_equal(v, v0)
    with pytest.raises(ValueError):
        with Engine(w) as e:
            e.snapshot_begin(np.empty(5))


def test_driver_checkpoints_hold_the_state(gpu, tmp_path):
    w = configs.ion_mixture_cfg(98, 2000)
    ctl = RunControl(nwgroup=1, nwsteps=6, ngroup=2, ntot=3, nind=2, nptensor=4, ncom=4, nckpt=5)
    seen = []
    with Engine(w) as e, Checkpointer(e, directory=str(tmp_path)) as ck:
        def hook(eng, istep, t, s):
            ck.checkpoint(eng, istep, t, s)
            ck._join()                               # the file is written; compare with the state
            x, v, _vo, _a = eng.get_state()
            seen.append((read_xvb(tmp_path / ck.written[-1]), x, v, t))
        run_md(e, ctl, on_checkpoint=hook)
    assert len(seen) >= 3
    for (fr,), x, v, t in seen:
        assert fr["ftype"] == "xv8b" and fr["n"] == w.n and fr["time"] == t
        assert np.array_equal(fr["x"], x) and np.array_equal(fr["v"], v)
        assert fr["sim_type"] == "ion-mixture"
