"""Vectorised numpy forces for a subset of target rows (test helper).

Used for parity checks at full benchmark sizes, where running the whole
O(N^2) oracle would take too long: the force on a sample of particles i is
summed over every j with the same formulas as the oracle (int_ion_pure.f,
int_ion_mix.f, int_nn.f), in numpy float64.
"""
import numpy as np

from yukawamd_b200 import abi


def min_image(d, L):
    d = np.where(d > L / 2, d - L, d)
    d = np.where(d < -L / 2, d + L, d)
    return d


def row_accels(p, x, zii, aii, rows):
    X = x.reshape(-1, 3)
    L = np.array(list(p.xl))
    n = len(X)
    out = np.zeros((len(rows), 3))
    for r, i in enumerate(rows):
        d = min_image(X[i] - X, L)
        r2 = (d * d).sum(1)
        mask = np.arange(n) != i
        if p.sim_type in (abi.YK_SIM_PURE_ION, abi.YK_SIM_ION_MIXTURE):
            m = mask & (r2 <= p.rccut ** 2)
            rr = np.sqrt(r2[m])
            fc = (1.0 + p.xmuc * rr) * np.exp(-p.xmuc * rr) / (rr * r2[m])
            if p.sim_type == abi.YK_SIM_ION_MIXTURE:
                fc = fc * zii[m]
            F = (fc[:, None] * d[m]).sum(0)
            if p.sim_type == abi.YK_SIM_PURE_ION:
                out[r] = p.frp * p.zi * p.zi * p.vc * F / (p.ai * p.xmass)
            else:
                fold = not (p.mix_mode == abi.YK_MIX_COMPAT and i == n - 1)
                F = zii[i] * F if fold else F
                out[r] = p.frp * p.vc * F / (aii[i] * p.xmass)
        else:
            f = np.zeros(n)
            if p.nuclear_on:
                m = mask & (r2 <= p.rncut ** 2)
                e = np.exp(-r2[m] / (2.0 * p.xpacket))
                B = np.where(zii[m] == zii[i], p.bb + p.cc, p.bb - p.cc)
                f[m] += (2.0 * p.aa * e + B) * e / p.xpacket
            if p.coulomb_on and zii[i] == 1.0:
                m = mask & (r2 <= p.rccut ** 2) & (zii == 1.0)
                rr = np.sqrt(r2[m])
                f[m] += p.vc * (1.0 + p.xmuc * rr) * np.exp(-p.xmuc * rr) / (rr * r2[m])
            out[r] = (f[:, None] * d).sum(0) / p.xmass
    return out
