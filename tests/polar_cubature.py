"""Independent high-accuracy cubature of the six kernel integrals of the
semi-analytic method (test infrastructure).

For a point x, a flat field triangle T and a time t, with r = |y - x| and
r_vec = y - x:
  ris1 = int_{T, c_S t < r < c_P t} 1/r             ris2 = same domain, r_i r_j / r^3
  ris3 = int_{T, c_S t < r < c_P t} 1/r^3           ris4 = same domain, r_i r_j / r^5
  ris5 = int_{T, r < c_S t} 1/r                     ris6 = same domain, r_i r_j / r^3
These are the quantities the reference evaluates in closed form
(functions/BEMenerg_indir/BEMenerg_core/BEMenerg_coreSA/calcoloMatrice/
BEMenerg_coreSA_calcMatrixSubBlock.m:88-97).  Here they are integrated in
polar coordinates about the projection of x on the plane of T: Gauss-Legendre
in the angle on sub-intervals cut at every vertex direction and every
front/edge crossing (so the integrand is smooth on each piece), and
Gauss-Legendre in the radius between the clipped limits.  Nothing of the
closed form is reused.
"""
from __future__ import annotations

import numpy as np

_GL = {}


def gl(n):
    if n not in _GL:
        _GL[n] = np.polynomial.legendre.leggauss(n)
    return _GL[n]


def _frame(T):
    P1, P2, P3 = T
    n = np.cross(P2 - P1, P3 - P1)
    n /= np.linalg.norm(n)
    u = (P2 - P1) / np.linalg.norm(P2 - P1)
    v = np.cross(n, u)
    return n, u, v


def _ray_limits(O2, V2, d):
    """Segment [s0, s1] of the ray O2 + s d (s >= 0) inside the convex 2-D
    triangle V2 (3 x 2, counter-clockwise)."""
    s0, s1 = 0.0, np.inf
    for k in range(3):
        a, b = V2[k], V2[(k + 1) % 3]
        e = b - a
        nin = np.array([-e[1], e[0]])          # inward normal for CCW order
        c0 = nin @ (O2 - a)
        c1 = nin @ d
        if abs(c1) < 1e-300:
            if c0 < 0:
                return 0.0, -1.0
            continue
        s = -c0 / c1
        if c1 > 0:
            s0 = max(s0, s)
        else:
            s1 = min(s1, s)
    return s0, s1


def _crossings(O2, V2, R):
    """Angles (about O2) where the circle of radius R meets the triangle edges."""
    out = []
    if R <= 0:
        return out
    for k in range(3):
        a, b = V2[k], V2[(k + 1) % 3]
        e = b - a
        w = a - O2
        A, B, C = e @ e, 2 * (w @ e), w @ w - R * R
        disc = B * B - 4 * A * C
        if disc < 0:
            continue
        for sg in (-1, 1):
            u = (-B + sg * np.sqrt(disc)) / (2 * A)
            if -1e-14 <= u <= 1 + 1e-14:
                p = w + u * e
                out.append(np.arctan2(p[1], p[0]))
    return out


def kernel_integrals(T, x, t, cP, cS, n_theta=24, n_rho=24, levels=3):
    """ris1..ris6 (6 x 3 x 3) by polar cubature; T is 3 x 3 (vertices)."""
    T = np.asarray(T, float)
    x = np.asarray(x, float)
    n, u, v = _frame(T)
    zeta_s = n @ (x - T[0])                  # signed height of x over the plane
    zeta = abs(zeta_s)
    O = x - zeta_s * n
    V2 = np.array([[(P - O) @ u, (P - O) @ v] for P in T])
    if np.cross(V2[1] - V2[0], V2[2] - V2[0]) < 0:
        V2 = V2[::-1]
    O2 = np.zeros(2)
    RP, RS = cP * t, cS * t
    rhoP = np.sqrt(max(RP * RP - zeta * zeta, 0.0))
    rhoS = np.sqrt(max(RS * RS - zeta * zeta, 0.0))
    # angular breakpoints
    br = [np.arctan2(p[1], p[0]) for p in V2]
    for R in (rhoP, rhoS):
        br += _crossings(O2, V2, R)
    br = np.unique(np.mod(np.array(br), 2 * np.pi))
    br = np.concatenate([br, [br[0] + 2 * np.pi]]) if len(br) else np.array([0.0, 2 * np.pi])
    if len(br) < 2:
        br = np.array([0.0, 2 * np.pi])
    xt, wt = gl(n_theta)
    xr, wr = gl(n_rho)
    out = np.zeros((6, 3, 3))

    def radial(d, lo, hi, kind):
        if hi <= lo:
            return np.zeros(6), np.zeros((6, 3, 3))
        rho = 0.5 * (hi - lo) * xr + 0.5 * (hi + lo)
        wq = 0.5 * (hi - lo) * wr * rho                  # rho d rho
        y = O[None, :] + rho[:, None] * (d[0] * u + d[1] * v)[None, :]
        rv = y - x[None, :]
        r = np.linalg.norm(rv, axis=1)
        rr = rv[:, :, None] * rv[:, None, :]
        sc = np.zeros(6)
        tn = np.zeros((6, 3, 3))
        if kind == "PS":       # between the fronts: ris1..ris4
            sc[0] = (wq / r).sum()
            tn[1] = (wq[:, None, None] * rr / r[:, None, None] ** 3).sum(0)
            sc[2] = (wq / r ** 3).sum()
            tn[3] = (wq[:, None, None] * rr / r[:, None, None] ** 5).sum(0)
        else:                  # inside the S front: ris5, ris6
            sc[4] = (wq / r).sum()
            tn[5] = (wq[:, None, None] * rr / r[:, None, None] ** 3).sum(0)
        return sc, tn

    def piece(a, b, depth):
        th = 0.5 * (b - a) * xt + 0.5 * (b + a)
        wth = 0.5 * (b - a) * wt
        acc = np.zeros((6, 3, 3))
        for thk, wk in zip(th, wth):
            d = np.array([np.cos(thk), np.sin(thk)])
            s0, s1 = _ray_limits(O2, V2, d)
            if s1 <= s0:
                continue
            sc1, tn1 = radial(d, max(s0, rhoS if RS > zeta else 0.0), min(s1, rhoP if RP > zeta else -1.0), "PS")
            sc2, tn2 = radial(d, s0, min(s1, rhoS if RS > zeta else -1.0), "S")
            tot = tn1 + tn2
            for m in (0, 2, 4):
                tot[m] += (sc1[m] + sc2[m]) * np.eye(3)
            acc += wk * tot
        return acc

    def adapt(a, b, depth):
        whole = piece(a, b, depth)
        if depth == 0:
            return whole
        mid = 0.5 * (a + b)
        halves = piece(a, mid, depth) + piece(mid, b, depth)
        scale = max(np.abs(halves).max(), 1e-300)
        if np.abs(halves - whole).max() <= 1e-13 * scale:
            return halves
        return adapt(a, mid, depth - 1) + adapt(mid, b, depth - 1)

    for a, b in zip(br[:-1], br[1:]):
        if b - a > 1e-15:
            out += adapt(a, b, levels)
    return out
