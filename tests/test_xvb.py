"""Revision-B configuration files (rw_xvb.f:36-203): record layout, round
trips for every file type and byte order, trajectories of several frames, and
the reference's file names (md_utils.f:31-34, 78-84)."""
import struct

import numpy as np
import pytest

from yukawamd_b200 import abi
from yukawamd_b200.xvb import (FTYPES, checkpoint_name, frame_bytes, read_xvb, save_config_name,
                               time_suffix, write_xvb)

WHEN = ("20261203", "101500.250", "+0100")


def _state(n, seed):
    rng = np.random.default_rng(seed)
    return rng.random(3 * n) * 50.0, rng.normal(size=3 * n) * 0.01, rng.normal(size=3 * n) * 1e-4


def _header():
    return {"time": 1234.5, "xl": [50.0, 51.0, 52.5], "ev": 27.9, "ek": 0.12, "px": 3.5e-4,
            "pp": [float(k) for k in range(1, 10)], "sim_type": abi.YK_SIM_ION_MIXTURE}


def test_record_layout_xv8b():
    n = 5
    x, v, _ = _state(n, 1)
    b = frame_bytes("xv8b", _header(), x, v, when=WHEN)
    off = 0
    lengths = []
    while off < len(b):
        (ln,) = struct.unpack("<i", b[off:off + 4])
        assert struct.unpack("<i", b[off + 4 + ln:off + 8 + ln])[0] == ln
        lengths.append(ln)
        off += ln + 8
    assert lengths == [6, 18, 23, 20, 16 * 8 + 4, 6 * 8 * n]
    assert b[4:10] == b"xv8b  "
    assert b[18:28] == b"MD        " and b[28:36] == b"6.2.0   "
    assert b[44:67] == b"20261203101500.250+0100"
    assert b[75:95] == b"ion-mixture         "
    vals = struct.unpack("<16di", b[103:103 + 132])
    assert vals[0] == 1234.5 and list(vals[1:4]) == [50.0, 51.0, 52.5] and vals[16] == n
    data = np.frombuffer(b[243:243 + 48 * n], dtype="<f8").reshape(n, 6)
    assert np.array_equal(data[:, :3].reshape(-1), x) and np.array_equal(data[:, 3:].reshape(-1), v)


@pytest.mark.parametrize("endian", ["<", ">"])
@pytest.mark.parametrize("ftype", FTYPES)
def test_round_trip(tmp_path, ftype, endian):
    n = 37
    x, v, a = _state(n, 2)
    path = tmp_path / ("c." + ftype)
    write_xvb(path, ftype, _header(), x, v, a, endian=endian, when=WHEN)
    (fr,) = read_xvb(path, endian=endian)
    assert fr["ftype"] == ftype and fr["n"] == n and fr["sim_type"] == "ion-mixture"
    assert fr["code_name"] == "MD" and fr["code_version"] == "6.2.0"
    assert fr["time"] == 1234.5 and fr["pp"] == [float(k) for k in range(1, 10)]
    if ftype in ("x4b", "xv4b"):
        assert np.array_equal(fr["x"], x.astype(np.float32).astype(np.float64))
    else:
        assert np.array_equal(fr["x"], x)
    if "v" in ftype:
        ref = v.astype(np.float32).astype(np.float64) if ftype == "xv4b" else v
        assert np.array_equal(fr["v"], ref)
    else:
        assert "v" not in fr
    if ftype == "xva8b":
        assert np.array_equal(fr["a"], a)


def test_trajectory_appends_frames(tmp_path):
    path = tmp_path / "md.traj.x8b"
    states = [_state(11, s) for s in range(3)]
    for k, (x, v, a) in enumerate(states):
        h = _header()
        h["time"] = 10.0 * k
        write_xvb(path, "x8b", h, x, append=k > 0, when=WHEN)
    frames = read_xvb(path)
    assert [f["time"] for f in frames] == [0.0, 10.0, 20.0]
    for f, (x, _v, _a) in zip(frames, states):
        assert np.array_equal(f["x"], x)


def test_corrupt_file_is_rejected(tmp_path):
    path = tmp_path / "bad.xv8b"
    x, v, _ = _state(4, 3)
    b = bytearray(frame_bytes("xv8b", _header(), x, v, when=WHEN))
    b[-1] ^= 0x40                          # break the trailing length marker
    path.write_bytes(bytes(b))
    with pytest.raises(ValueError):
        read_xvb(path)


def test_names_follow_md_utils():
    assert time_suffix(1234.5) == "00000001235"           # nint rounds halves away from zero
    assert time_suffix(2500000.25) == "00002500000"
    assert checkpoint_name(1234.4) == "md.00000001234.xv8b"
    assert save_config_name(99.0, "xv8b", append=False) == "md.00000000099.xv8b"
    assert save_config_name(99.0, "x4b", append=True, tend=5000.0) == "md.traj.00000005000.x4b"


def test_bad_ftype_and_missing_velocities():
    x, v, _ = _state(3, 4)
    with pytest.raises(ValueError):
        frame_bytes("xv9b", _header(), x, v)
    with pytest.raises(ValueError):
        frame_bytes("xv8b", _header(), x)
