"""Generate tests/golden/kat.json: known-answer cases at 50 significant digits.

The reference (MD 6.2.0) ships no tests, golden vectors or fixtures, and its
Fortran cannot be compiled here, so the CPU restatement in oracle/ is pinned by
these cases instead.  They are written independently of the oracle's C code,
straight from the physics the reference implements:

  pure ion  (int_ion_pure.f:98-254)  F_ij = frp zi^2 vc (1+mu r) e^{-mu r}/r^3 d_ij
  mixture   (int_ion_mix.f:105-295)  same with Z_i Z_j, and the compat-mode
                                     omission of Z_{n-1} on particle n-1
  nucleon   (int_nn.f:130-345)       HPP Gaussians + p-p screened Coulomb
  Verlet    (vel_verlet_1/2/3.f)     one step of each integrator with the
                                     'B-field' force case (a = 0 + Lorentz)

with the minimum image by the reference's conditional +/-L rule, the energy
shift evcut when r_c <= |L|/2, and the scaling/unpacking of accel's tail.
Inputs are exact binary64 values; outputs are 50-digit decimals rounded to
the nearest double in the JSON.

Run:  python tests/golden/make_kat.py   (rewrites kat.json next to it)
"""
import json
import os
from decimal import Decimal as D, getcontext

import numpy as np

getcontext().prec = 50

HBARC = 197.327
ALPHA = 1.0 / 137.036
VC = ALPHA * HBARC
XMASS = 931.0


def dd(x):
    return D(float(x))


def min_image(xi, xj, xl):
    out = []
    for k in range(3):
        d = xi[k] - xj[k]
        if d > xl[k] / 2:
            d = d - xl[k]
        if d < -xl[k] / 2:
            d = d + xl[k]
        out.append(d)
    return out


def evcut_of(p, scale):
    xl = [dd(v) for v in p["xl"]]
    rccut = dd(p["rccut"])
    half_diag = (xl[0] ** 2 + xl[1] ** 2 + xl[2] ** 2).sqrt() / 2
    if rccut <= half_diag:
        return scale * (-(dd(p["xmuc"]) * rccut)).exp() / rccut
    return D(0)


def accel_exact(p, x, zii, aii, do_meas):
    """Exact forces, packed raw sums and scalars for one accel call."""
    n = len(zii)
    xl = [dd(v) for v in p["xl"]]
    X = [[dd(x[3 * i + k]) for k in range(3)] for i in range(n)]
    Z = [dd(z) for z in zii]
    A = [dd(a) for a in aii]
    mu = dd(p["xmuc"])
    rc2 = dd(p["rccut"]) ** 2
    st = p["sim_type"]
    F = [[D(0)] * 3 for _ in range(n)]
    U = D(0)
    W = D(0)
    P = [D(0)] * 6       # xx xy xz yy yz zz
    if st in (2, 3):
        evcut = evcut_of(p, D(1))
        for i in range(n):
            for j in range(i + 1, n):
                d = min_image(X[i], X[j], xl)
                r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2]
                if r2 > rc2:
                    continue
                r = r2.sqrt()
                e = (-(mu * r)).exp()
                w = Z[i] * Z[j] if st == 3 else D(1)
                u = e / r - evcut
                f = (1 + mu * r) * e / (r * r2)
                U += w * u
                W += w * f * r2
                for k in range(3):
                    F[i][k] += Z[j] * f * d[k] if st == 3 else f * d[k]
                    F[j][k] -= Z[i] * f * d[k] if st == 3 else f * d[k]
                dd_ = [d[0] * d[0], d[0] * d[1], d[0] * d[2], d[1] * d[1], d[1] * d[2], d[2] * d[2]]
                for k in range(6):
                    P[k] += w * f * dd_[k]
        if st == 3:
            for i in range(n):
                if i == n - 1 and p.get("mix_mode", 0) == 0:
                    continue          # compat: the i loop ends at n-2
                for k in range(3):
                    F[i][k] *= Z[i]
            C = dd(p["frp"]) * dd(p["vc"])
            acc = [[C * F[i][k] / (A[i] * dd(p["xmass"])) for k in range(3)] for i in range(n)]
        else:
            C = dd(p["frp"]) * dd(p["zi"]) * dd(p["zi"]) * dd(p["vc"])
            acc = [[C * F[i][k] / (dd(p["ai"]) * dd(p["xmass"])) for k in range(3)] for i in range(n)]
    elif st == 1:
        vc = dd(p["vc"])
        evcut = evcut_of(p, vc)
        lam = dd(p["xpacket"])
        rn2 = dd(p["rncut"]) ** 2
        aa, bb, cc = dd(p["aa"]), dd(p["bb"]), dd(p["cc"])
        for i in range(n):
            for j in range(i + 1, n):
                d = min_image(X[i], X[j], xl)
                r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2]
                f = D(0)
                hit = False
                if p["nuclear_on"] and r2 <= rn2:
                    e = (-(r2 / (2 * lam))).exp()
                    B = bb + cc if Z[i] == Z[j] else bb - cc
                    U += (aa * e + B) * e
                    fn = (2 * aa * e + B) * e / lam
                    W += fn * r2
                    f += fn
                    hit = True
                if p["coulomb_on"] and r2 <= rc2 and Z[i] == 1 and Z[j] == 1:
                    r = r2.sqrt()
                    e = (-(mu * r)).exp()
                    U += vc * e / r - evcut
                    fc = vc * (1 + mu * r) * e / (r * r2)
                    W += fc * r2
                    f += fc
                    hit = True
                if hit:
                    for k in range(3):
                        F[i][k] += f * d[k]
                        F[j][k] -= f * d[k]
                    dd_ = [d[0] * d[0], d[0] * d[1], d[0] * d[2], d[1] * d[1], d[1] * d[2], d[2] * d[2]]
                    for k in range(6):
                        P[k] += f * dd_[k]
        C = D(1)
        acc = [[F[i][k] / dd(p["xmass"]) for k in range(3)] for i in range(n)]
    else:
        raise ValueError(st)
    if not do_meas:
        U, W, P = D(0), D(0), [D(0)] * 6
    a = [acc[i][k] for i in range(n) for k in range(3)]
    a += [U, W, D(0), P[0], P[1], P[2], P[3], P[4], P[5]]
    if do_meas:
        ev = C * U / n
        vir = C * W
        px = dd(p["rho"]) * (dd(p["kT"]) + vir / (3 * n))
        pu = [C * v for v in P]
        pp = [pu[0], pu[1], pu[2], pu[1], pu[3], pu[4], pu[2], pu[4], pu[5]]
    else:
        ev = vir = px = D(0)
        pp = [D(0)] * 9
    return a, dict(ev=ev, vir=vir, px=px, pp=pp)


def lorentz_omega(p, z, a, literal):
    return literal * dd(z) * dd(p["bfield"]) / dd(a)


def verlet_exact(p, x, v, a, zii, aii, do_meas, integ):
    """One step of vel_verlet_<integ> with the B-field force case (accel sets
    a = 0 and leaves ev/pp untouched, so they enter as zero here)."""
    n = len(zii)
    xl = [dd(t) for t in p["xl"]]
    dt = dd(p["dt"])
    X = [dd(t) for t in x]
    V = [dd(t) for t in v]
    Aa = [dd(t) for t in a[:3 * n]]
    xm = dd(p["xmass"])
    for i in range(n):
        for k in range(3):
            e = 3 * i + k
            X[e] = X[e] + V[e] * dt + dt * dt / 2 * Aa[e]
            if X[e] < 0:
                X[e] += xl[k]
            if X[e] > xl[k]:
                X[e] -= xl[k]
    VOLD = list(V)
    if integ == 2:
        V = [V[e] + dt * Aa[e] for e in range(3 * n)]
        Anew = [D(0)] * (3 * n)
        if p["bfield"] != 0.0:
            for i in range(n):
                om = lorentz_omega(p, zii[i], aii[i], D("3.218404e-20"))
                Anew[3 * i] = Anew[3 * i] + V[3 * i + 1] * om
                Anew[3 * i + 1] = Anew[3 * i + 1] - V[3 * i] * om
        V = [(V[e] + (VOLD[e] + dt * Anew[e])) / 2 for e in range(3 * n)]
    elif integ == 1:
        V = [V[e] + dt / 2 * Aa[e] for e in range(3 * n)]
        Anew = [D(0)] * (3 * n)
        V = [V[e] + dt / 2 * Anew[e] for e in range(3 * n)]
    else:
        lit = dd(np.float32(3.218404e-20))
        h = dt / 2
        for i in range(n):
            om = lorentz_omega(p, zii[i], aii[i], lit)
            w = h * om
            a1, a2, a3 = Aa[3 * i], Aa[3 * i + 1], Aa[3 * i + 2]
            V[3 * i] = (1 - w * w) * V[3 * i] + 2 * w * V[3 * i + 1] + h * (a1 + w * a2)
            V[3 * i + 1] = (1 - w * w) * V[3 * i + 1] - 2 * w * V[3 * i] + h * (a2 - w * a1)
            V[3 * i + 2] = V[3 * i + 2] + h * a3
        Anew = [D(0)] * (3 * n)
        for i in range(n):
            om = lorentz_omega(p, zii[i], aii[i], lit)
            w = h * om
            V[3 * i] = V[3 * i] / (1 + w * w)
            V[3 * i + 1] = V[3 * i + 1] / (1 + w * w)
    measure = do_meas or integ in (1, 3)
    if measure:
        s = [D(0)] * 6
        for i in range(n):
            vi = V[3 * i:3 * i + 3]
            ai = dd(aii[i])
            s[0] += ai * vi[0] * vi[0]
            s[1] += ai * vi[0] * vi[1]
            s[2] += ai * vi[0] * vi[2]
            s[3] += ai * vi[1] * vi[1]
            s[4] += ai * vi[1] * vi[2]
            s[5] += ai * vi[2] * vi[2]
        ek = xm / 2 * (s[0] + s[3] + s[5]) / n
        vol = xl[0] * xl[1] * xl[2]
        pk = [xm * t / vol for t in s]
        pp = [pk[0], pk[1], pk[2], pk[1], pk[3], pk[4], pk[2], pk[4], pk[5]]
    else:
        ek = D(0)
        pp = [D(0)] * 9
    out = dict(x=X, v=V, a=Anew, ek=ek, pp=pp)
    if integ == 2:
        out["vold"] = VOLD
    return out


def base_params(**kw):
    p = dict(sim_type=2, precision=0, integrator=2, mix_mode=0, coulomb_on=1,
             nuclear_on=0, xl=[100.0, 100.0, 100.0], rccut=1e50, rncut=0.0,
             xmuc=0.1, vc=VC, frp=1.0, xmass=XMASS, rho=1e-4, kT=0.05, dt=5.0,
             bfield=0.0, zi=8.0, ai=16.0, aa=110.0, bb=-26.0, cc=24.0,
             xpacket=1.25, time=0.0)
    p.update(kw)
    return p


def rncut_default():
    import math
    xpacket, aa, bb, cc = 1.25, 110.0, -26.0, 24.0
    xeps = (math.sqrt(2.0 * xpacket) / (2.0 * (-bb + cc))) * 0.0001 * 2.0 ** -53
    r = math.sqrt(-math.log((-bb - cc) / (2.0 * aa)))
    r0, step = r, 1.0
    while True:
        while r * math.exp(-(r * r)) > xeps:
            r0, r = r, r + step
        if step < 0.11:
            break
        step, r = step / 10.0, r0
    return r * math.sqrt(2.0 * xpacket)


def cases():
    out = []
    rng = np.random.default_rng(20121217)
    # pure ion, 2 particles across the x face, r_c below the half diagonal
    p = base_params(xl=[100.0, 120.0, 90.0], rccut=40.0, xmuc=0.0625)
    x = np.array([1.5, 60.0, 45.0, 97.25, 62.5, 44.0])
    out.append(("pure2_face", p, x, [8.0, 8.0], [16.0, 16.0]))
    # pure ion, 3 collinear along y: one pair beyond the cutoff
    p = base_params(xl=[100.0, 100.0, 100.0], rccut=30.0, xmuc=0.05)
    x = np.array([50.0, 10.0, 50.0, 50.0, 35.0, 50.0, 50.0, 75.0, 50.0])
    out.append(("pure3_collinear", p, x, [8.0] * 3, [16.0] * 3))
    # pure ion, 17 random particles, cutoff below the half diagonal
    L = [70.0, 70.0, 70.0]
    x = (rng.random((17, 3)) * np.array(L)).reshape(-1)
    p = base_params(xl=L, rccut=30.0, xmuc=1.0 / 14.9, zi=6.0, ai=12.0, rho=17 / 70.0 ** 3)
    out.append(("pure17_random", p, x, [6.0] * 17, [12.0] * 17))
    # ion mixture, 6 particles, three species, no cutoff (evcut = 0)
    L = [50.0, 55.0, 60.0]
    x = (rng.random((6, 3)) * np.array(L)).reshape(-1)
    z = [6.0, 8.0, 26.0, 8.0, 6.0, 26.0]
    for mode, name in ((0, "mix6_compat"), (1, "mix6_fixed")):
        p = base_params(sim_type=3, xl=L, rccut=1e50, xmuc=1.0 / 29.85, mix_mode=mode,
                        rho=6 / (50.0 * 55.0 * 60.0))
        out.append((name, p, x, z, [2.0 * t for t in z]))
    # ion mixture with a cutoff below the half diagonal
    L = [40.0, 40.0, 40.0]
    x = (rng.random((9, 3)) * np.array(L)).reshape(-1)
    z = [6.0, 8.0, 26.0, 8.0, 8.0, 8.0, 6.0, 26.0, 8.0]
    p = base_params(sim_type=3, xl=L, rccut=18.0, xmuc=0.07, rho=9 / 40.0 ** 3)
    out.append(("mix9_cut", p, x, z, [2.0 * t for t in z]))
    # nucleon: 4 p + 4 n in a small box, HPP + p-p Coulomb (rccut default)
    L = [12.0, 12.0, 12.0]
    x = (rng.random((8, 3)) * np.array(L)).reshape(-1)
    z = [1.0, 0.0, 1.0, 0.0, 1.0, 0.0, 1.0, 0.0]
    p = base_params(sim_type=1, xl=L, rccut=1e50, rncut=rncut_default(), xmuc=0.1,
                    nuclear_on=1, coulomb_on=1, rho=8 / 12.0 ** 3, kT=1.0, dt=2.0)
    out.append(("nn8_box12", p, x, z, [1.0] * 8))
    # nucleon: larger box so rncut and a finite rccut both bite
    L = [30.0, 30.0, 30.0]
    x = (rng.random((12, 3)) * np.array(L)).reshape(-1)
    z = [float(t) for t in (rng.random(12) < 0.5)]
    z[0] = z[1] = 1.0
    p = base_params(sim_type=1, xl=L, rccut=14.0, rncut=rncut_default(), xmuc=0.1,
                    nuclear_on=1, coulomb_on=1, rho=12 / 30.0 ** 3, kT=1.0, dt=2.0)
    out.append(("nn12_cut", p, x, z, [1.0] * 12))
    return out


def verlet_cases():
    rng = np.random.default_rng(7)
    n = 4
    L = [20.0, 20.0, 20.0]
    x = (rng.random((n, 3)) * np.array(L)).reshape(-1)
    x[0] = 0.01                       # drifts across the lower face
    x[4] = 19.995                     # drifts across the upper face
    v = rng.standard_normal(3 * n) * 0.01
    v[0] = -0.003
    v[4] = 0.004
    a = rng.standard_normal(3 * n) * 1e-4
    z = [6.0, 8.0, 26.0, 1.0]
    am = [12.0, 16.0, 52.0, 1.0]
    out = []
    for integ in (1, 2, 3):
        for bf in (0.0, 2.0e17):
            p = base_params(sim_type=4, integrator=integ, xl=L, dt=2.0, bfield=bf)
            out.append(("verlet%d_b%s" % (integ, "on" if bf else "off"), p, x, v, a, z, am))
    return out


def fmt(vals):
    return [float(t) for t in vals]


def main():
    doc = {"generator": "tests/golden/make_kat.py", "digits": 50, "accel": [], "verlet": []}
    for name, p, x, z, am in cases():
        for meas in (True, False):
            a, s = accel_exact(p, x, z, am, meas)
            doc["accel"].append(dict(name=name, do_meas=meas, params=p, x=fmt(x), zii=fmt(z),
                                     aii=fmt(am), a=fmt(a), ev=float(s["ev"]), vir=float(s["vir"]),
                                     px=float(s["px"]), pp=fmt(s["pp"])))
    for name, p, x, v, a, z, am in verlet_cases():
        for meas in (True, False):
            o = verlet_exact(p, x, v, a, z, am, meas, p["integrator"])
            rec = dict(name=name, do_meas=meas, params=p, x0=fmt(x), v0=fmt(v), a0=fmt(a),
                       zii=fmt(z), aii=fmt(am), x=fmt(o["x"]), v=fmt(o["v"]), a=fmt(o["a"]),
                       ek=float(o["ek"]), pp=fmt(o["pp"]))
            if "vold" in o:
                rec["vold"] = fmt(o["vold"])
            doc["verlet"].append(rec)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "kat.json")
    with open(path, "w") as f:
        json.dump(doc, f, indent=1)
    print("wrote", path, len(doc["accel"]), "accel cases,", len(doc["verlet"]), "verlet cases")


if __name__ == "__main__":
    main()
