"""ctypes wrapper of the CPU restatement (TEST INFRASTRUCTURE ONLY).

Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg and
reference arm, as the checker or the timed CPU baseline.  The engine never
imports it.  Parity unpinned by reference outputs; pinned by the 50-digit
known-answer cases in tests/golden/.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from yukawamd_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS = {"double": "liborc.so", "long_double": "liborc_ld.so"}
_cache = {}

_dp = C.POINTER(C.c_double)


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _ptr(arr):
    if arr is None:
        return None
    assert arr.dtype == np.float64 and arr.flags["C_CONTIGUOUS"]
    return arr.ctypes.data_as(_dp)


def _load(variant):
    if variant in _cache:
        return _cache[variant]
    path = os.path.join(HERE, _LIBS[variant])
    if not os.path.exists(path):
        build()
    lib = C.CDLL(path)
    P = C.POINTER(abi.YkParams)
    S = C.POINTER(abi.YkScalars)
    lib.orc_accel.argtypes = [P, C.c_int, _dp, _dp, _dp, C.c_int, _dp, S]
    lib.orc_newton.argtypes = [P, C.c_int, _dp, _dp, _dp, _dp, _dp, _dp, C.c_int, S]
    lib.orc_ttot.argtypes = [P, C.c_int, _dp, _dp]
    lib.orc_ttot.restype = C.c_double
    lib.orc_tnorm.argtypes = [P, C.c_int, _dp, _dp]
    lib.orc_cancel_vcom.argtypes = [P, C.c_int, _dp, _dp]
    lib.orc_strain.argtypes = [P, C.c_int, _dp, _dp, _dp, _dp]
    lib.orc_rncut.argtypes = [C.c_double] * 4
    lib.orc_rncut.restype = C.c_double
    lib.orc_thomas_fermi_xmuc.argtypes = [C.c_double, C.c_double, C.c_int]
    lib.orc_thomas_fermi_xmuc.restype = C.c_double
    lib.orc_vtot.argtypes = [P, C.c_int, _dp, _dp, _dp, _dp]
    lib.orc_gofr_counts.argtypes = [P, C.c_int, _dp, C.c_int, _dp]
    lib.orc_set_threads.argtypes = [C.c_int]
    lib.orc_set_row_range.argtypes = [C.c_int, C.c_int]
    lib.orc_max_threads.restype = C.c_int
    lib.orc_long_double_accum.restype = C.c_int
    _cache[variant] = lib
    return lib


def _f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


def _arrays(params, n, zii, aii):
    """The reference keeps zii/aii arrays for every sim type; fill them for
    pure-ion runs from zi/ai when the caller passes None."""
    if zii is None:
        zii = np.full(n, params.zi)
    if aii is None:
        aii = np.full(n, params.ai if params.ai else 1.0)
    return _f64(zii), _f64(aii)


class Oracle:
    def __init__(self, variant="double", threads=1):
        self.lib = _load(variant)
        self.variant = variant
        self.set_threads(threads)

    def set_threads(self, threads):
        self.lib.orc_set_threads(int(threads))
        self.threads = int(threads)

    def set_row_range(self, i0=0, i1=0x7fffffff):
        self.lib.orc_set_row_range(int(i0), int(i1))

    def accel(self, params, x, zii=None, aii=None, do_meas=True, scalars=None):
        x = _f64(x)
        n = len(x) // 3
        zii, aii = _arrays(params, n, zii, aii)
        a = np.zeros(3 * (n + 3))
        s = scalars if scalars is not None else abi.YkScalars()
        rc = self.lib.orc_accel(C.byref(params), n, _ptr(x), _ptr(zii), _ptr(aii),
                                int(bool(do_meas)), _ptr(a), C.byref(s))
        if rc:
            raise RuntimeError("orc_accel failed: %s" % abi.STATUS_NAMES.get(rc, rc))
        return a, s

    def newton(self, params, x, v, vold, a, zii=None, aii=None, do_meas=True,
               scalars=None):
        """In-place step on x, v, vold (double[3n]) and a (double[3(n+3)])."""
        n = len(x) // 3
        zii, aii = _arrays(params, n, zii, aii)
        s = scalars if scalars is not None else abi.YkScalars()
        rc = self.lib.orc_newton(C.byref(params), n, _ptr(x), _ptr(v), _ptr(vold),
                                 _ptr(a), _ptr(zii), _ptr(aii), int(bool(do_meas)),
                                 C.byref(s))
        if rc:
            raise RuntimeError("orc_newton failed: %s" % abi.STATUS_NAMES.get(rc, rc))
        return s

    def ttot(self, params, v, aii):
        v, aii = _f64(v), _f64(aii)
        return self.lib.orc_ttot(C.byref(params), len(aii), _ptr(v), _ptr(aii))

    def tnorm(self, params, v, aii):
        self.lib.orc_tnorm(C.byref(params), len(aii), _ptr(v), _ptr(_f64(aii)))

    def cancel_vcom(self, params, v, aii):
        self.lib.orc_cancel_vcom(C.byref(params), len(aii), _ptr(v), _ptr(_f64(aii)))

    def strain(self, params, x, xl, xl0, deps):
        self.lib.orc_strain(C.byref(params), len(x) // 3, _ptr(x), _ptr(xl),
                            _ptr(_f64(xl0)), _ptr(_f64(deps)))

    def rncut(self, aa=110.0, bb=-26.0, cc=24.0, xpacket=1.25):
        return self.lib.orc_rncut(aa, bb, cc, xpacket)

    def thomas_fermi_xmuc(self, ztot, rho, n):
        return self.lib.orc_thomas_fermi_xmuc(ztot, rho, n)

    def gofr_counts(self, params, x, nbin):
        x = _f64(x)
        counts = np.zeros(nbin)
        rc = self.lib.orc_gofr_counts(C.byref(params), len(x) // 3, _ptr(x), int(nbin), _ptr(counts))
        if rc:
            raise RuntimeError("orc_gofr_counts failed")
        return counts

    def vtot(self, params, x, zii=None):
        x = _f64(x)
        n = len(x) // 3
        zii = _f64(zii) if zii is not None else np.full(n, params.zi)
        ev = C.c_double()
        pr = C.c_double()
        rc = self.lib.orc_vtot(C.byref(params), n, _ptr(x), _ptr(zii),
                               C.byref(ev), C.byref(pr))
        if rc:
            raise RuntimeError("orc_vtot failed")
        return ev.value, pr.value
