"""The C-ABI library: loads, exports every declared entry point, struct layouts
match, host-side argument checks.  No compute calls (no GPU needed)."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from yukawamd_b200 import _lib, abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "yukawa_engine.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^YK_API [^(]*?\b(yk_\w+)\(", text, flags=re.M)))


def test_library_loads_and_exports_every_symbol():
    h = _lib.lib()
    names = declared_symbols()
    assert len(names) >= 14
    for name in names:
        assert hasattr(h, name), name
    assert set(names) == set(_lib.SIGNATURES)


def test_exported_dynamic_symbols():
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH],
                         capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r" T (yk_\w+)", out))
    assert set(declared_symbols()) <= exported


def test_struct_layouts_match_c(tmp_path):
    src = tmp_path / "sz.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "yukawa_engine.h"\n'
                   'int main(void){printf("%zu %zu %zu %zu %zu\\n", sizeof(yk_params),'
                   ' sizeof(yk_scalars), offsetof(yk_params, xl), offsetof(yk_params, time),'
                   ' offsetof(yk_scalars, time)); return 0;}\n')
    exe = tmp_path / "sz"
    subprocess.run(["/usr/bin/gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True)
    vals = [int(t) for t in subprocess.run([str(exe)], capture_output=True, text=True,
                                           check=True).stdout.split()]
    assert vals == [C.sizeof(abi.YkParams), C.sizeof(abi.YkScalars),
                    abi.YkParams.xl.offset, abi.YkParams.time.offset,
                    abi.YkScalars.time.offset]


def test_params_default_matches_reference_defaults():
    h = _lib.lib()
    p = abi.YkParams()
    assert h.yk_params_default(C.byref(p)) == abi.YK_OK
    q = abi.default_params()
    for name, _ in abi.YkParams._fields_:
        a, b = getattr(p, name), getattr(q, name)
        if name == "xl":
            assert list(a) == list(b)
        else:
            assert a == b, name
    assert p.vc == pytest.approx(1.439964, rel=1e-6)     # ALPHA*HBARC
    assert p.rccut == 1e50 and p.xmass == 931.0


def _create(p, x, v=None, zii=None, aii=None, n=None):
    h = _lib.lib()
    ctx = C.c_void_p()
    dp = C.POINTER(C.c_double)
    f = lambda a: None if a is None else a.ctypes.data_as(dp)  # noqa: E731
    n = len(x) // 3 if n is None else n
    rc = h.yk_create(C.byref(p), n, f(x), f(v), f(zii), f(aii), C.byref(ctx))
    if rc == abi.YK_OK:
        h.yk_destroy(ctx)
    return rc, h.yk_last_error(None).decode()


def _params():
    p = abi.default_params()
    for k in range(3):
        p.xl[k] = 10.0
    p.dt = 1.0
    p.zi, p.ai = 8.0, 16.0
    return p


def test_create_rejects_bad_arguments_on_host():
    x = np.random.default_rng(0).random(30) * 10
    rc, msg = _create(_params(), x, n=0)
    assert rc == abi.YK_ERR_ARG and "n must be" in msg
    p = _params()
    p.dt = 0.0
    assert _create(p, x)[0] == abi.YK_ERR_ARG
    p = _params()
    p.xl[1] = -1.0
    assert _create(p, x)[0] == abi.YK_ERR_ARG
    p = _params()
    p.sim_type = 9
    assert _create(p, x)[0] == abi.YK_ERR_ARG
    p = _params()
    p.sim_type = abi.YK_SIM_ION_MIXTURE
    assert _create(p, x)[0] == abi.YK_ERR_ARG          # needs zii / aii
    bad = x.copy()
    bad[4] = np.nan
    assert _create(_params(), bad)[0] == abi.YK_ERR_NONFINITE
    badv = np.zeros(30)
    badv[0] = np.inf
    assert _create(_params(), x, v=badv)[0] == abi.YK_ERR_NONFINITE


def test_null_context_is_an_error_not_a_crash():
    h = _lib.lib()
    s = abi.YkScalars()
    assert h.yk_accel(None, 1, None, C.byref(s)) == abi.YK_ERR_ARG
    assert h.yk_newton(None, 0, C.byref(s)) == abi.YK_ERR_ARG
    assert h.yk_run(None, 3, 0, None) == abi.YK_ERR_ARG
    assert h.yk_destroy(None) == abi.YK_ERR_ARG
    assert h.yk_last_error(None)


def test_version_string():
    assert b"sm_100a" in _lib.lib().yk_version()
