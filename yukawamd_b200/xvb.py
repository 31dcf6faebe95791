"""Revision-B binary configuration files (rw_xvb.f:36-203) and the
checkpoint / save_config writers of md_utils.f:19-114.

A file is a sequence of Fortran unformatted sequential records: each record
is its payload framed by a 4-byte length before and after.  One frame
(configuration) is six records (rw_xvb.f:174-197):

  1  ftype                     character*6
  2  code_name, code_version   character*10, character*8   ('MD', '6.2.0')
  3  date, daytime, timezone   character*8, *10, *5        (date_and_time)
  4  sim_type                  character*20
  5  time, xl(1:3), ev, ek, px, pp(3,3), n
                               11 real*8 + pp column-major (9 real*8) + integer*4
  6  the data, per particle i = 0..n-1:
       x4b   x(1:3,i) as real*4        xv4b  x(1:3,i), v(1:3,i) as real*4
       x8b   x(1:3,i) as real*8        xv8b  x(1:3,i), v(1:3,i) as real*8
       xva8b x(1:3,i), v(1:3,i), a(1:3,i) as real*8

Character fields are blank-padded.  Byte order is the writer's: gfortran
builds (mdef/Ubuntu.def) write little-endian, the Intel builds
(mdef/Quarry.def:22, -convert big_endian) big-endian; `endian` selects it
for both the markers and the data.  Records are limited to 2**31 - 1 bytes
(n < 44.7 million for xv8b): larger records would need the compiler's
subrecord scheme, which is not written.

`Checkpointer` takes a snapshot of the engine state asynchronously
(yk_snapshot_begin: device copy on the engine's stream, host copy on a side
stream) and writes the file on a background thread, so checkpoints overlap
the following steps.
"""
import datetime
import math
import struct
import threading

import numpy as np

from . import abi

FTYPES = ("x4b", "xv4b", "x8b", "xv8b", "xva8b")
CODE_NAME = "MD"
CODE_VERSION = "6.2.0"
SIM_NAMES = {abi.YK_SIM_NUCLEON: "nucleon", abi.YK_SIM_PURE_ION: "pure-ion",
             abi.YK_SIM_ION_MIXTURE: "ion-mixture", abi.YK_SIM_BFIELD: "B-field"}
MAX_RECORD = 2 ** 31 - 1


def _chars(s, width):
    b = s.encode("ascii")[:width]
    return b + b" " * (width - len(b))


def _record(payload, endian):
    if len(payload) > MAX_RECORD:
        raise ValueError("record of %d bytes exceeds 2**31 - 1" % len(payload))
    m = struct.pack(endian + "i", len(payload))
    return m + payload + m


def date_and_time(now=None):
    """Fortran date_and_time: 'CCYYMMDD', 'hhmmss.sss', '+hhmm'."""
    now = now or datetime.datetime.now().astimezone()
    off = now.utcoffset() or datetime.timedelta(0)
    mins = int(off.total_seconds()) // 60
    sign = "+" if mins >= 0 else "-"
    mins = abs(mins)
    return (now.strftime("%Y%m%d"), now.strftime("%H%M%S") + ".%03d" % (now.microsecond // 1000),
            "%s%02d%02d" % (sign, mins // 60, mins % 60))


def frame_bytes(ftype, header, x, v=None, a=None, endian="<", when=None):
    """One configuration as bytes.  header: dict with time, xl (3), ev, ek, px,
    pp (9 values, pp(1,1) pp(2,1) pp(3,1) pp(1,2) ... column-major, as the
    engine's yk_scalars.pp), sim_type (name or YK_SIM_* code)."""
    ftype = ftype.strip()
    if ftype not in FTYPES:
        raise ValueError("unknown Rev.B file type %r" % ftype)
    x = np.asarray(x, dtype=np.float64).reshape(-1, 3)
    n = x.shape[0]
    cols = [x]
    if ftype in ("xv4b", "xv8b", "xva8b"):
        if v is None:
            raise ValueError("%s needs velocities" % ftype)
        cols.append(np.asarray(v, dtype=np.float64).reshape(n, 3))
    if ftype == "xva8b":
        if a is None:
            raise ValueError("xva8b needs accelerations")
        cols.append(np.asarray(a, dtype=np.float64)[:3 * n].reshape(n, 3))
    data = np.concatenate(cols, axis=1)
    dt = (endian + "f4") if ftype in ("x4b", "xv4b") else (endian + "f8")
    payload = np.ascontiguousarray(data.astype(dt)).tobytes()
    sim = header.get("sim_type", "")
    if not isinstance(sim, str):
        sim = SIM_NAMES[int(sim)]
    d, t, z = when or date_and_time()
    pp = list(header.get("pp", [0.0] * 9))
    vals = [header["time"]] + list(header["xl"]) + [header.get("ev", 0.0), header.get("ek", 0.0),
                                                   header.get("px", 0.0)] + pp
    out = [_record(_chars(ftype, 6), endian),
           _record(_chars(CODE_NAME, 10) + _chars(CODE_VERSION, 8), endian),
           _record(_chars(d, 8) + _chars(t, 10) + _chars(z, 5), endian),
           _record(_chars(sim, 20), endian),
           _record(struct.pack(endian + "16d", *vals) + struct.pack(endian + "i", n), endian),
           _record(payload, endian)]
    return b"".join(out)


def write_xvb(path, ftype, header, x, v=None, a=None, append=False, endian="<", when=None):
    """write_xvb (rw_xvb.f:148-203): one frame, appended or in a new file."""
    with open(path, "ab" if append else "wb") as f:
        f.write(frame_bytes(ftype, header, x, v, a, endian, when))


def _read_record(f, endian):
    m = f.read(4)
    if not m:
        return None
    if len(m) < 4:
        raise ValueError("truncated record marker")
    (ln,) = struct.unpack(endian + "i", m)
    if ln < 0:
        raise ValueError("subrecords (records over 2**31 - 1 bytes) are not supported")
    payload = f.read(ln)
    tail = f.read(4)
    if len(payload) != ln or len(tail) != 4 or struct.unpack(endian + "i", tail)[0] != ln:
        raise ValueError("corrupt record (length markers disagree)")
    return payload


def read_xvb(path, endian="<"):
    """read_xvb (rw_xvb.f:36-144) for every frame of a file.  Returns a list of
    dicts: ftype, code_name, code_version, date, daytime, timezone, sim_type,
    time, xl, ev, ek, px, pp (9, column-major), n, x, and v / a as present."""
    frames = []
    with open(path, "rb") as f:
        while True:
            r = _read_record(f, endian)
            if r is None:
                break
            fr = {"ftype": r.decode("ascii").strip()}
            r = _read_record(f, endian)
            fr["code_name"], fr["code_version"] = r[:10].decode().strip(), r[10:18].decode().strip()
            r = _read_record(f, endian)
            fr["date"], fr["daytime"], fr["timezone"] = r[:8].decode(), r[8:18].decode(), r[18:23].decode()
            fr["sim_type"] = _read_record(f, endian).decode("ascii").strip()
            r = _read_record(f, endian)
            vals = struct.unpack(endian + "16d", r[:128])
            (n,) = struct.unpack(endian + "i", r[128:132])
            fr.update(time=vals[0], xl=list(vals[1:4]), ev=vals[4], ek=vals[5], px=vals[6],
                      pp=list(vals[7:16]), n=n)
            r = _read_record(f, endian)
            ft = fr["ftype"]
            ncol = {"x4b": 3, "xv4b": 6, "x8b": 3, "xv8b": 6, "xva8b": 9}[ft]
            dt = (endian + "f4") if ft in ("x4b", "xv4b") else (endian + "f8")
            data = np.frombuffer(r, dtype=dt).reshape(n, ncol).astype(np.float64)
            fr["x"] = data[:, 0:3].reshape(-1).copy()
            if ncol >= 6:
                fr["v"] = data[:, 3:6].reshape(-1).copy()
            if ncol == 9:
                fr["a"] = data[:, 6:9].reshape(-1).copy()
            frames.append(fr)
    return frames


def _nint(x):
    """Fortran nint: nearest integer, halves away from zero."""
    return int(math.floor(x + 0.5)) if x >= 0 else -int(math.floor(-x + 0.5))


def time_suffix(t):
    """The i5.5,i6.6 time stamp md_utils.f:32-33 builds from a time in fm/c."""
    return "%05d%06d" % (int(t / 1000000.0), _nint(math.fmod(t, 1000000.0)))


def checkpoint_name(t):
    """md.<time>.xv8b (md_utils.f:31-34)."""
    return "md.%s.xv8b" % time_suffix(t)


def save_config_name(t, ftype, append, tend=None):
    """md.traj.<tend>.<ftype> when appending, else md.<time>.<ftype> (md_utils.f:78-84)."""
    if append:
        return "md.traj.%s.%s" % (time_suffix(tend if tend is not None else t), ftype.strip())
    return "md.%s.%s" % (time_suffix(t), ftype.strip())


def header_from(engine, t, scalars):
    """The header globals md.F holds when it checkpoints: time, xl and the
    last step's ev, ek, px, pp (zeros after a non-measuring step)."""
    s = scalars
    return {"time": t, "xl": list(engine.params.xl), "sim_type": int(engine.params.sim_type),
            "ev": s.ev if s is not None else 0.0, "ek": s.ek if s is not None else 0.0,
            "px": s.px if s is not None else 0.0,
            "pp": list(s.pp) if s is not None else [0.0] * 9}


class Checkpointer:
    """Checkpoint / save_config hooks for yukawamd_b200.driver.run_md.

    Each call starts an asynchronous snapshot into one of two page-locked host
    buffer sets and hands the file write to a background thread; the engine
    goes on stepping meanwhile.  close() (or leaving the with-block) waits
    for every pending write.  Files go to `directory` under the reference's
    names; `ftype` and `append` are save_config's (md_globals.f:89-98)."""

    def __init__(self, engine, directory=".", ftype="xv8b", append=True, tend=None, endian="<"):
        from .engine import host_register
        self.engine = engine
        self.dir = directory
        self.ftype = ftype
        self.append = append
        self.tend = tend
        self.endian = endian
        n3 = 3 * engine.n
        self._bufs = [tuple(np.empty(n3) for _ in range(3)) for _ in range(2)]
        for bs in self._bufs:
            for b in bs:
                host_register(b)
        self._turn = 0
        self._thread = None
        self._lock = threading.Lock()
        self.written = []

    def _start(self, path, ftype, header, append):
        import os
        self._join()
        x, v, a = self._bufs[self._turn]
        self._turn ^= 1
        need_a = ftype == "xva8b"
        self.engine.snapshot_begin(x, v, a if need_a else None)
        eng = self.engine

        def work():
            eng.snapshot_wait()
            write_xvb(os.path.join(self.dir, path), ftype, header, x, v, a if need_a else None,
                      append=append, endian=self.endian)
            with self._lock:
                self.written.append(path)

        # the previous write has finished (_join above), so the background
        # thread is the only one that waits on this snapshot
        self._thread = threading.Thread(target=work)
        self._thread.start()

    def _join(self):
        if self._thread is not None:
            self._thread.join()
            self._thread = None

    def checkpoint(self, engine, istep, t, scalars):
        """md_utils.f:19-38: xv8b of x and v, one file per checkpoint."""
        self._start(checkpoint_name(t), "xv8b", header_from(engine, t, scalars), False)

    def save_config(self, engine, istep, t, scalars):
        """md_utils.f:61-114 for the Rev.B types."""
        self._start(save_config_name(t, self.ftype, self.append, self.tend), self.ftype,
                    header_from(engine, t, scalars), self.append)

    def close(self):
        from .engine import host_unregister
        self._join()
        for bs in self._bufs:
            for b in bs:
                host_unregister(b)
        self._bufs = []

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
