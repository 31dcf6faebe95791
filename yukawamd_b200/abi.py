"""ctypes mirror of include/yukawa_engine.h (structs and constants).

The field order and types must match the C header exactly; tests check the
struct sizes against the C library (``yk_abi_sizes``).
"""
import ctypes as C

YK_OK = 0
YK_ERR_ARG = 1
YK_ERR_CUDA = 2
YK_ERR_NOMEM = 3
YK_ERR_STATE = 4
YK_ERR_TIMEOUT = 5
YK_ERR_NONFINITE = 6
YK_ERR_UNSUPPORTED = 7

STATUS_NAMES = {
    YK_OK: "YK_OK", YK_ERR_ARG: "YK_ERR_ARG", YK_ERR_CUDA: "YK_ERR_CUDA",
    YK_ERR_NOMEM: "YK_ERR_NOMEM", YK_ERR_STATE: "YK_ERR_STATE",
    YK_ERR_TIMEOUT: "YK_ERR_TIMEOUT", YK_ERR_NONFINITE: "YK_ERR_NONFINITE",
    YK_ERR_UNSUPPORTED: "YK_ERR_UNSUPPORTED",
}

# accel's select case (int_control.f:69-87)
YK_SIM_NUCLEON = 1
YK_SIM_PURE_ION = 2
YK_SIM_ION_MIXTURE = 3
YK_SIM_BFIELD = 4

SIM_TYPE_NAMES = {
    "nucleon": YK_SIM_NUCLEON,
    "pure-ion": YK_SIM_PURE_ION,
    "ion-mixture": YK_SIM_ION_MIXTURE,
    "B-field": YK_SIM_BFIELD,
}

YK_PREC_FP64 = 0
YK_PREC_MIXED = 1

YK_VV1 = 1
YK_VV2 = 2
YK_VV3 = 3

YK_MIX_COMPAT = 0
YK_MIX_FIXED = 1

# md_globals.f:24-28, 122
HBARC = 197.327
ALPHA = 1.0 / 137.036
ME = 0.510999
PI = 3.14159265358979324
VC = ALPHA * HBARC
XMASS = 931.00


class YkParams(C.Structure):
    _fields_ = [
        ("sim_type", C.c_int),
        ("precision", C.c_int),
        ("integrator", C.c_int),
        ("mix_mode", C.c_int),
        ("coulomb_on", C.c_int),
        ("nuclear_on", C.c_int),
        ("device", C.c_int),
        ("reserved0", C.c_int),
        ("xl", C.c_double * 3),
        ("rccut", C.c_double),
        ("rncut", C.c_double),
        ("xmuc", C.c_double),
        ("vc", C.c_double),
        ("frp", C.c_double),
        ("xmass", C.c_double),
        ("rho", C.c_double),
        ("kT", C.c_double),
        ("dt", C.c_double),
        ("bfield", C.c_double),
        ("zi", C.c_double),
        ("ai", C.c_double),
        ("aa", C.c_double),
        ("bb", C.c_double),
        ("cc", C.c_double),
        ("xpacket", C.c_double),
        ("time", C.c_double),
    ]

    def as_dict(self):
        d = {}
        for name, _ in self._fields_:
            val = getattr(self, name)
            d[name] = list(val) if name == "xl" else val
        return d


class YkScalars(C.Structure):
    _fields_ = [
        ("ev", C.c_double),
        ("vir", C.c_double),
        ("px", C.c_double),
        ("ek", C.c_double),
        ("pp", C.c_double * 9),
        ("time", C.c_double),
    ]

    def as_dict(self):
        return {"ev": self.ev, "vir": self.vir, "px": self.px, "ek": self.ek,
                "pp": list(self.pp), "time": self.time}


class YkTuning(C.Structure):
    _fields_ = [
        ("force_kernel", C.c_int),
        ("pair_seg", C.c_int),
        ("sort_every", C.c_int),
        ("graph_steps", C.c_int),
        ("source_split", C.c_int),
        ("targets_per_thread", C.c_int),
    ]


KERNEL_AUTO = 0
KERNEL_ROWS = 1
KERNEL_PAIRS = 2
KERNEL_NEAR = 3


class YkPerf(C.Structure):
    _fields_ = [
        ("run_ms", C.c_double),
        ("force_ms", C.c_double),
        ("steps", C.c_longlong),
        ("force_calls", C.c_longlong),
    ]


def default_params():
    """Reference defaults of md_globals.f:36-140 (same values as
    yk_params_default in the C library)."""
    p = YkParams()
    p.sim_type = YK_SIM_PURE_ION
    p.precision = YK_PREC_FP64
    p.integrator = YK_VV2
    p.mix_mode = YK_MIX_COMPAT
    p.coulomb_on = 1
    p.nuclear_on = 0
    p.device = 0
    p.rccut = 1.0e50
    p.rncut = 0.0
    p.xmuc = 0.0
    p.vc = VC
    p.frp = 1.0
    p.xmass = XMASS
    p.xpacket = 1.25
    p.aa = 110.0
    p.bb = -26.0
    p.cc = 24.0
    return p
