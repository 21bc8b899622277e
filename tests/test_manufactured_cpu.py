"""The reference's manufactured case 'TEST' (BEMenerg_core_calcNucleoTn.m:13-132:
the boundary value on the screen [-1,1]^2 whose solution is the constant
density phi = (1, 1, 1)), the only known answer the reference defines for the
indirect path.  The oracle's cubature of the TEST integrals is checked
against scipy's adaptive integration of the reference's integrand, then the
oracle's semi-analytic assembly with that right-hand side must march to
phi = (1, 1, 1): since sum_{l<=n} E_l 1 telescopes to the first time
difference of the single layer of the constant density, which is the TEST
value, b_n = sum_{l<=n} E_l 1 holds up to rounding."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

from elastodynamicebem_b200 import mesh, problem  # noqa: E402


def _f(r1, r2, t, cP, cS):
    """f_c of one instant (the nucl_c of the reference regrouped by instant),
    with I_P - I_S taken as (1/c_S^2 - 1/c_P^2)/(2r) where both fronts passed."""
    r = np.hypot(r1, r2)
    if t <= 0:
        return np.zeros(3)
    hP = 1.0 if t - r / cP > 0 else 0.0
    hS = 1.0 if t - r / cS > 0 else 0.0
    JP, JS = hP / (cP ** 2 * r), hS / (cS ** 2 * r)
    if hS:
        B = (1 / cS ** 2 - 1 / cP ** 2) / (2 * r)
    elif hP:
        B = (t - r / cP) * (t + r / cP) / (2 * r ** 3)
    else:
        B = 0.0
    A = JP - JS
    c2, s2, cs = r1 * r1 / (r * r), r2 * r2 / (r * r), r1 * r2 / (r * r)
    return np.array([A * c2 + B * (3 * c2 - 1) + JS + cs * (A + 3 * B),
                     A * s2 + B * (3 * s2 - 1) + JS + cs * (A + 3 * B), JS - B])


def _adaptive(x1, x2, t0, t1, prm):
    from scipy import integrate
    cP, cS = prm.velP, prm.velS
    radii = [v * t for t in (t0, t1) if t > 0 for v in (cS, cP)]
    out = []
    for comp in range(3):
        def g(y1, y2):
            return (_f(y1 - x1, y2 - x2, t1, cP, cS) - _f(y1 - x1, y2 - x2, t0, cP, cS))[comp]

        def opt_in(y2):
            pts = [x1] + [x1 + sg * np.sqrt(rho ** 2 - (y2 - x2) ** 2) for rho in radii if rho > abs(y2 - x2)
                          for sg in (-1, 1)]
            return {"points": [p for p in pts if -1 < p < 1], "limit": 200, "epsabs": 1e-13, "epsrel": 1e-11}
        pts = [x2] + [x2 + sg * rho for rho in radii for sg in (-1, 1)]
        opt_out = {"points": [p for p in pts if -1 < p < 1], "limit": 200, "epsabs": 1e-12, "epsrel": 1e-10}
        v, _ = integrate.nquad(g, [[-1, 1], [-1, 1]], opts=[opt_in, opt_out])
        out.append(v / (4 * np.pi * prm.rho))
    return np.array(out)


@pytest.mark.parametrize("case", [(0.3, -0.7, 0.25, 0.3), (-0.45, 0.6, 0.0, 0.1)])
def test_oracle_cubature_against_adaptive(case):
    prm = problem.ProblemParams(1.0, 1.0, 2.0, 1.0, 20)
    ref = _adaptive(*case, prm)
    got = O.tn_test(*case, prm)
    assert np.abs(got - ref).max() <= 1e-10 * np.abs(ref).max()


def test_oracle_cubature_converged():
    prm = problem.ProblemParams(1.0, 1.0, 2.0, 1.0, 20)
    for case in [(0.1, 0.2, 0.0, 0.05), (-0.9, 0.95, 0.5, 0.55), (0.0, 0.0, 0.9, 0.95)]:
        a = O.tn_test(*case, prm)
        b = O.tn_test(*case, prm, nang=40, nsplit=8, nrad=40)
        assert np.abs(a - b).max() <= 1e-14


@pytest.mark.parametrize("n", [2, 4])
def test_known_answer_oracle(n):
    """Oracle SA assembly + TEST right-hand side + LU marching: phi = (1,1,1)."""
    m = mesh.screen_uniform(n, half=1.0)
    prm = problem.ProblemParams(1.0, 1.0, 2.0, 1.0, 10)
    L = O.num_blocks(m, prm)
    E, _ = O.assemble_sa(m, prm, 7, 0, L)
    b = O.rhs(m, prm, 7, problem.DATUM_TEST)
    ones = np.ones(E.shape[1])
    rows = [E[l] @ ones for l in range(L)] + [np.zeros_like(ones)] * max(0, prm.nT - L)
    S = np.cumsum(np.stack(rows), axis=0)[:prm.nT].T
    assert np.linalg.norm(b - S) <= 1e-10 * np.linalg.norm(S)
    phi = O.march(E, b)
    assert np.abs(phi - 1).max() <= 1e-9
