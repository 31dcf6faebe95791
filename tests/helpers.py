"""Shared helpers for the tests (parameter building, error norms)."""
import numpy as np

from yukawamd_b200 import abi


def params_from_dict(d):
    p = abi.default_params()
    for k, v in d.items():
        if k == "xl":
            for i in range(3):
                p.xl[i] = float(v[i])
        else:
            setattr(p, k, v)
    return p


def rel_norm(a, b):
    """||a - b||_2 / ||b||_2 (0 if both are zero)."""
    a = np.asarray(a, dtype=float)
    b = np.asarray(b, dtype=float)
    nb = np.linalg.norm(b)
    if nb == 0.0:
        return float(np.linalg.norm(a))
    return float(np.linalg.norm(a - b) / nb)


def rel(a, b):
    if b == 0.0:
        return abs(a)
    return abs(a - b) / abs(b)


def scalars_vec(s):
    return np.array([s.ev, s.vir, s.px, s.ek] + list(s.pp))
