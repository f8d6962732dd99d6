"""Generate tests/golden/known_answers.json: known-answer vectors for the Euler flux routines.

The reference (jmark/nemo, Fortran) has no tests and no golden vectors and cannot be compiled in
this environment.  These vectors come from a second, independent restatement of the reference's
formulas written here in plain Python (math module, no numpy), so that the C++ oracle is checked
against code that shares nothing with it but the published formulas:
  xflux            source/equations/euler/equations_mod.f90:64-79
  logmean          source/equations/euler/two_point/chandrashekar/two_point_flux_mod.f90:13-32
  Chandrashekar    same file :34-77
  Rusanov          source/equations/euler/riemann/rusanov/riemann_mod.f90:7-24
  HLLC/HLLE hybrid source/equations/euler/riemann/hllc/riemann_mod.f90:7-104
y/z directions rotate (rho, m_y, m_z, m_x, E) into x and back, as the reference's wrappers do.
Run: python tests/golden/make_golden.py
"""
import json
import math
import os
import random

K = 1.4


def pres(u):
    return (K - 1) * (u[4] - 0.5 / u[0] * (u[1] ** 2 + u[2] ** 2 + u[3] ** 2))


def xflux(u):
    p, vx = pres(u), u[1] / u[0]
    return [u[1], vx * u[1] + p, vx * u[2], vx * u[3], vx * (u[4] + p)]


def rot(d, u):
    return list(u) if d == 0 else ([u[0], u[2], u[3], u[1], u[4]] if d == 1 else [u[0], u[3], u[1], u[2], u[4]])


def unrot(d, f):
    return list(f) if d == 0 else ([f[0], f[3], f[1], f[2], f[4]] if d == 1 else [f[0], f[2], f[3], f[1], f[4]])


def logmean(a, b):
    x = a / b
    if abs(a - b) < 1e-4:
        u = (x * (x - 2) + 1) / (x * (x + 2) + 1)
        return (a + b) * (0.5 - u * (1 / 6 - u * (2 / 45 - 22 / 945 * u)))
    return (a - b) / math.log(x)


def chandra(u, v):
    bu, bv = 0.5 * u[0] / pres(u), 0.5 * v[0] / pres(v)
    uu = [u[i] / u[0] for i in (1, 2, 3)]
    vv = [v[i] / v[0] for i in (1, 2, 3)]
    dens = logmean(u[0], v[0])
    vel = [0.5 * (a + b) for a, b in zip(uu, vv)]
    p = 0.5 * (u[0] + v[0]) / (bu + bv)
    h = 0.5 / (K - 1) / logmean(bu, bv) + p / dens + sum(c * c for c in vel) - 0.25 * sum(
        a * a + b * b for a, b in zip(uu, vv))
    f0 = dens * vel[0]
    return [f0, f0 * vel[0] + p, f0 * vel[1], f0 * vel[2], f0 * h]


def lam(u):
    return abs(u[1] / u[0]) + math.sqrt(K * pres(u) / u[0])


def rusanov(uL, uR):
    fl, fr, lm = xflux(uL), xflux(uR), max(lam(uL), lam(uR))
    return [0.5 * (a + b + lm * (c - d)) for a, b, c, d in zip(fl, fr, uL, uR)]


def hllc(UL, UR):
    beta = math.sqrt(0.5 * (K - 1) / K)
    VL, VR = UL[1] / UL[0], UR[1] / UR[0]
    pL, pR = pres(UL), pres(UR)
    cL, cR = math.sqrt(K * pL / UL[0]), math.sqrt(K * pR / UR[0])
    HL, HR = (UL[4] + pL) / UL[0], (UR[4] + pR) / UR[0]
    sl, sr = math.sqrt(UL[0]), math.sqrt(UR[0])
    Ht = (sl * HL + sr * HR) / (sl + sr)
    vt = (sl * VL + sr * VR) / (sl + sr)
    at = math.sqrt((K - 1) * (Ht - 0.5 * vt ** 2))
    SL = min(vt - at, VL - beta * cL, 0.0)
    SR = max(vt + at, VR + beta * cR, 0.0)
    if SL >= 0:
        return xflux(UL)
    if SR <= 0:
        return xflux(UR)
    FL, FR = xflux(UL), xflux(UR)
    sm = math.sqrt(abs(pL - pR) / (pL + pR))
    FH = [(SR * a - SL * b + SL * SR * (c - d)) / (SR - SL) for a, b, c, d in zip(FL, FR, UR, UL)]
    SS = (pR - pL + UL[1] * (SL - VL) - UR[1] * (SR - VR)) / (UL[0] * (SL - VL) - UR[0] * (SR - VR))
    if SL <= 0 <= SS:
        U, F, S, V, p = UL, FL, SL, VL, pL
    else:
        U, F, S, V, p = UR, FR, SR, VR, pR
    Q = U[0] * (S - V) / (S - SS)
    Us = [Q, Q * SS, Q * U[2] / U[0], Q * U[3] / U[0], Q * (U[4] / U[0] + (SS - V) * (SS + p / U[0] / (S - V)))]
    return [sm * fh + (1 - sm) * (f + S * (us - uu)) for fh, f, us, uu in zip(FH, F, Us, U)]


def cons(rho, vx, vy, vz, p):
    return [rho, rho * vx, rho * vy, rho * vz, p / (K - 1) + 0.5 * rho * (vx * vx + vy * vy + vz * vz)]


def main():
    rng = random.Random(20240611)
    states = [cons(1.0, 0.0, 0.0, 0.0, 1.0), cons(0.125, 0.0, 0.0, 0.0, 0.1), cons(1.0, 0.75, -0.3, 0.2, 1.0)]
    for _ in range(6):
        states.append(cons(rng.uniform(0.2, 3), rng.uniform(-2, 2), rng.uniform(-2, 2), rng.uniform(-2, 2),
                           rng.uniform(0.05, 5)))
    out = {"kappa": K, "flux": [], "logmean": [], "rusanov": [], "hllc": [], "chandrashekar": []}
    for u in states:
        for d in range(3):
            out["flux"].append({"dir": d, "u": u, "f": unrot(d, xflux(rot(d, u)))})
    for a, b in [(1.0, 1.5), (0.3, 0.30005), (2.0, 7.0), (1.0, 1.0 + 9.9e-5), (5e4, 5.0001e4)]:
        out["logmean"].append({"a": a, "b": b, "r": logmean(a, b)})
    for i in range(len(states)):
        for j in range(len(states)):
            if i == j:
                continue
            uL, uR = states[i], states[j]
            for d in range(3):
                out["rusanov"].append({"dir": d, "uL": uL, "uR": uR, "f": unrot(d, rusanov(rot(d, uL), rot(d, uR)))})
                out["hllc"].append({"dir": d, "uL": uL, "uR": uR, "f": unrot(d, hllc(rot(d, uL), rot(d, uR)))})
                out["chandrashekar"].append({"dir": d, "u": uL, "v": uR, "f": unrot(d, chandra(rot(d, uL), rot(d, uR)))})
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "known_answers.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=0)
    print(path)


if __name__ == "__main__":
    main()
