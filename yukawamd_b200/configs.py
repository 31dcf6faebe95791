"""Seeded synthetic inputs for the engine.

The reference builds its initial state in input1.F / initconfig.f from a
namelist: positions uniform in the box (initconfig.f:203-219), Maxwell
velocities scaled by sqrt(kT/(A*xmass)) (initconfig.f:362-374) followed by
cancel_vcom and tnorm (gen_utils.f:64-110), and the derived parameters of
input1.F:260-322 (screening length, automatic nuclear cutoff).  The reference
ships no datasets; every workload here is generated from a numpy PCG64 seed
that is recorded with the run.

Workloads (one per benchmark configuration of the engine):
  pure_ion_ocp      N=4,096 pure-ion OCP, Z=8, A=16, kappa=1, Gamma=175
  ion_mixture       N=55,296 mixture Z={6,8,26} fractions {0.2,0.7,0.1},
                    kappa=0.5, effective Gamma=150
  nucleon_matter    N=51,200 nucleons, proton fraction 0.4, n_B=0.05 fm^-3,
                    kT=1 MeV, HPP nuclear + p-p screened Coulomb (lambda=10 fm)
  replica_ensemble  256 pure-ion boxes, N log-uniform in [1e3, 2e4],
                    Gamma U[50,250], kappa U[0.5,2], Z in {6,8,26}
  request_stream    Poisson arrivals of runs for the serving loop
"""
from dataclasses import dataclass, field
import math

import numpy as np

from . import abi

ION_DENSITY = 7.18e-5        # ions / fm^3, the ion benchmarks' density


def rncut_auto(aa=110.0, bb=-26.0, cc=24.0, xpacket=1.25):
    """Automatic HPP cutoff of input1.F:296-311: the radius where the force
    has fallen to 2**-53 of Fmin = 1e-4, stepped in 1, 0.1, ... decrements."""
    xepsilon = (math.sqrt(2.0 * xpacket) / (2.0 * (-bb + cc))) * 0.0001 * 2.0 ** -53
    rncut = math.sqrt(-math.log((-bb - cc) / (2.0 * aa)))
    rncut0 = rncut
    xdeltar = 1.0
    while True:
        while rncut * math.exp(-(rncut * rncut)) > xepsilon:
            rncut0 = rncut
            rncut = rncut + xdeltar
        if xdeltar < 0.11:
            break
        xdeltar = xdeltar / 10.0
        rncut = rncut0
    return rncut * math.sqrt(2.0 * xpacket)


def thomas_fermi_xmuc(ztot, rho, n):
    """Thomas-Fermi inverse screening length of input1.F:266-278."""
    rhoe = (ztot * rho) / n
    xkf = (3.0 * abi.PI ** 2 * rhoe) ** (1.0 / 3.0) * abi.HBARC
    ef = math.sqrt(xkf ** 2 + abi.ME ** 2)
    qtf = 2.0 * math.sqrt((abi.ALPHA / abi.PI) * xkf * ef)
    return qtf / abi.HBARC


def cancel_vcom_tnorm(v, aii, kT, xmass=abi.XMASS):
    """Zero total momentum, then rescale to eka = 1.5 kT (gen_utils.f:64-110)."""
    v = v.reshape(-1, 3)
    vcom = (aii[:, None] * v).sum(0) / aii.sum()
    v = v - vcom
    eka = 0.5 * xmass * float((aii * (v * v).sum(1)).sum()) / len(aii)
    if eka > 0.0:                   # a single particle has no thermal motion left
        v = v / math.sqrt(eka / (1.5 * kT))
    return v.reshape(-1)


@dataclass
class Workload:
    """One engine run: parameters plus initial arrays in the Fortran layout."""
    name: str
    params: dict
    x: np.ndarray            # double[3n]
    v: np.ndarray            # double[3n]
    zii: np.ndarray          # double[n]
    aii: np.ndarray          # double[n]
    steps: int = 100
    seed: int = 0
    notes: dict = field(default_factory=dict)

    @property
    def n(self):
        return len(self.zii)

    @property
    def pairs_per_step(self):
        n = self.n
        return n * (n - 1) // 2

    def yk_params(self, **overrides):
        p = abi.default_params()
        d = dict(self.params)
        d.update(overrides)
        for k, val in d.items():
            if k == "xl":
                for i in range(3):
                    p.xl[i] = float(val[i])
            else:
                setattr(p, k, val)
        return p


def _box_and_positions(rng, n, density):
    length = (n / density) ** (1.0 / 3.0)
    x = rng.random((n, 3)) * length
    return length, x.reshape(-1)


def _maxwell(rng, aii, kT, xmass=abi.XMASS):
    velfac = np.sqrt(kT / (aii * xmass))
    v = rng.standard_normal((len(aii), 3)) * velfac[:, None]
    return cancel_vcom_tnorm(v.reshape(-1), aii, kT, xmass)


def plasma_frequency(density, z, a, vc=abi.VC, xmass=abi.XMASS):
    """omega_p = sqrt(4 pi n Z^2 vc / (A xmass)) in c/fm; z, a may be arrays of
    per-particle values (then the mixture average of Z^2/A is used)."""
    z = np.asarray(z, dtype=float)
    a = np.asarray(a, dtype=float)
    return math.sqrt(4.0 * math.pi * density * float(np.mean(z * z / a)) * vc / xmass)


def pure_ion(n, z, a, kappa, gamma, seed, density=ION_DENSITY, dt_wp=0.02,
             steps=100, name="pure_ion"):
    """Pure-ion Yukawa OCP: Gamma = Z^2 vc / (a kT), a = (3/(4 pi n))^(1/3),
    lambda = a/kappa, r_c = min(L/2, 10 lambda), dt = dt_wp / omega_p."""
    rng = np.random.default_rng(np.random.PCG64(seed))
    length, x = _box_and_positions(rng, n, density)
    a_ws = (3.0 / (4.0 * math.pi * density)) ** (1.0 / 3.0)
    lam = a_ws / kappa
    kT = z * z * abi.VC / (a_ws * gamma)
    zii = np.full(n, float(z))
    aii = np.full(n, float(a))
    v = _maxwell(rng, aii, kT)
    wp = plasma_frequency(density, zii[:1], aii[:1])
    params = dict(sim_type=abi.YK_SIM_PURE_ION, xl=[length] * 3,
                  rccut=min(length / 2.0, 10.0 * lam), xmuc=1.0 / lam,
                  rho=n / length ** 3, kT=kT, dt=dt_wp / wp, zi=float(z),
                  ai=float(a), coulomb_on=1, nuclear_on=0)
    return Workload(name, params, x, v, zii, aii, steps, seed,
                    dict(L=length, a_ws=a_ws, lam=lam, gamma=gamma,
                         kappa=kappa, omega_p=wp))


def ion_mixture(n, zs, fracs, kappa, gamma_eff, seed, density=ION_DENSITY,
                dt_wp=0.02, steps=10000, name="ion_mixture"):
    """Ion mixture, A = 2Z, species drawn per particle with the given number
    fractions.  Gamma_eff = <Z^(5/3)> vc / (a_e kT) with a_e the electron-sphere
    radius, n_e = <Z> n (nominal fractions); lambda = a/kappa with a the ion
    sphere radius; dt = dt_wp / omega_p of the mixture."""
    rng = np.random.default_rng(np.random.PCG64(seed))
    length, x = _box_and_positions(rng, n, density)
    zs = np.asarray(zs, dtype=float)
    fracs = np.asarray(fracs, dtype=float)
    zii = zs[rng.choice(len(zs), size=n, p=fracs / fracs.sum())]
    aii = 2.0 * zii
    a_ws = (3.0 / (4.0 * math.pi * density)) ** (1.0 / 3.0)
    lam = a_ws / kappa
    zbar = float((fracs * zs).sum() / fracs.sum())
    z53 = float((fracs * zs ** (5.0 / 3.0)).sum() / fracs.sum())
    a_e = (3.0 / (4.0 * math.pi * zbar * density)) ** (1.0 / 3.0)
    kT = z53 * abi.VC / (a_e * gamma_eff)
    v = _maxwell(rng, aii, kT)
    wp = plasma_frequency(density, zii, aii)
    params = dict(sim_type=abi.YK_SIM_ION_MIXTURE, xl=[length] * 3,
                  rccut=min(length / 2.0, 10.0 * lam), xmuc=1.0 / lam,
                  rho=n / length ** 3, kT=kT, dt=dt_wp / wp,
                  coulomb_on=1, nuclear_on=0)
    return Workload(name, params, x, v, zii, aii, steps, seed,
                    dict(L=length, a_ws=a_ws, a_e=a_e, lam=lam,
                         gamma_eff=gamma_eff, kappa=kappa, omega_p=wp))


def nucleon(n, xp, n_b, kT, lam, dt, seed, steps=10000, name="nucleon"):
    """Nucleon matter (int_nn.f): zii = 1 for protons, 0 for neutrons,
    aii = 1; HPP defaults (md_globals.f:127-130); rncut automatic; screened
    p-p Coulomb with xmuc = 1/lambda and rccut at its 1e50 default."""
    rng = np.random.default_rng(np.random.PCG64(seed))
    length, x = _box_and_positions(rng, n, n_b)
    nprot = int(round(xp * n))
    zii = np.zeros(n)
    zii[rng.permutation(n)[:nprot]] = 1.0
    aii = np.ones(n)
    v = _maxwell(rng, aii, kT)
    params = dict(sim_type=abi.YK_SIM_NUCLEON, xl=[length] * 3,
                  rccut=1.0e50, rncut=rncut_auto(), xmuc=1.0 / lam,
                  rho=n / length ** 3, kT=kT, dt=dt, coulomb_on=1,
                  nuclear_on=1)
    return Workload(name, params, x, v, zii, aii, steps, seed,
                    dict(L=length, nprot=nprot, lam=lam))


# ---- the benchmark workloads -------------------------------------------

def pure_ion_ocp(seed=1, n=4096):
    return pure_ion(n, 8, 16, kappa=1.0, gamma=175.0, seed=seed, steps=100,
                    name="pure-ion OCP N=%d" % n)


def ion_mixture_cfg(seed=2, n=55296):
    return ion_mixture(n, [6, 8, 26], [0.2, 0.7, 0.1], kappa=0.5,
                       gamma_eff=150.0, seed=seed, steps=10000,
                       name="ion-mixture N=%d" % n)


def nucleon_matter(seed=3, n=51200):
    return nucleon(n, 0.4, 0.05, 1.0, 10.0, 2.0, seed=seed, steps=10000,
                   name="nucleon N=%d" % n)


def replica_ensemble(seed=4, count=256, nmin=1000, nmax=20000):
    rng = np.random.default_rng(np.random.PCG64(seed))
    out = []
    for r in range(count):
        n = int(round(math.exp(rng.uniform(math.log(nmin), math.log(nmax)))))
        gamma = float(rng.uniform(50.0, 250.0))
        kappa = float(rng.uniform(0.5, 2.0))
        z = int(rng.choice([6, 8, 26]))
        out.append(pure_ion(n, z, 2 * z, kappa, gamma,
                            seed=int(rng.integers(1 << 31)), steps=1000,
                            name="replica %d" % r))
    return out


def request_stream(seed=5, count=64, rate_per_s=4.0, nmin=512, nmax=131072,
                   smin=100, smax=5000):
    """Poisson arrivals: 70% ion runs (half pure, half mixture), 30% nucleon.
    Returns a list of (arrival_time_s, Workload)."""
    rng = np.random.default_rng(np.random.PCG64(seed))
    t = 0.0
    out = []
    for k in range(count):
        t += float(rng.exponential(1.0 / rate_per_s))
        n = int(round(math.exp(rng.uniform(math.log(nmin), math.log(nmax)))))
        steps = int(rng.integers(smin, smax + 1))
        s = int(rng.integers(1 << 31))
        u = float(rng.random())
        if u < 0.35:
            z = int(rng.choice([6, 8, 26]))
            w = pure_ion(n, z, 2 * z, float(rng.uniform(0.5, 2.0)),
                         float(rng.uniform(50.0, 250.0)), seed=s, steps=steps,
                         name="req%d pure-ion" % k)
        elif u < 0.70:
            w = ion_mixture(n, [6, 8, 26], [0.2, 0.7, 0.1],
                            float(rng.uniform(0.5, 2.0)),
                            float(rng.uniform(50.0, 250.0)), seed=s,
                            steps=steps, name="req%d ion-mixture" % k)
        else:
            w = nucleon(n, 0.4, 0.05, 1.0, 10.0, 2.0, seed=s, steps=steps,
                        name="req%d nucleon" % k)
        w.steps = steps
        out.append((t, w))
    return out
