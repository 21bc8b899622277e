"""The closed-form post-processing skips the instants at which the P front
cannot have reached a triangle (``pp_reach`` in csrc/march.cu): the centroid
distance less the longest edge, less a margin of half the longest edge and
the projection's tolerances.  These checks evaluate the oracle's single-point
case split (the restatement of BEMenerg_postProcA_singlePoint.m and of the
projection in preparazioneTriangolo.m / calcoloDistanzaTriangolo.m) at
instants just below that bound and at random instants below it, on meshes
whose tolerances matter differently (unit scale, a 1e-3 scale where the
1e-6 edge tolerance is large against the edges, a 1e3 scale, graded
slivers), with points in the triangles' planes, near their vertices and
edges, and off them: every skipped instant must be one where the closed form
finds no front (case 0), so that the skipped block is exactly zero."""
import numpy as np
import pytest

from elastodynamicebem_b200 import mesh as M


def reach(T, x):
    """The bound of pp_reach (same formula, host rounding)."""
    V0, V1, V2 = T
    nn = np.cross(V0 - V2, V1 - V2)
    area = np.linalg.norm(nn) / 2
    ctr = (V0 + V1 + V2) / 3
    maxL = max(np.linalg.norm(V0 - V1), np.linalg.norm(V1 - V2), np.linalg.norm(V0 - V2))
    r = np.linalg.norm(x - ctr)
    tol = 0.5 * maxL + 1e-5 + (1e-6 * maxL / area if area > 0 else np.inf) + 1e-12 * r
    return r - maxL - tol


def _meshes():
    s = M.screen_uniform(4)
    yield "sphere80", M.icosphere(1)
    yield "screen32_small", M.Mesh(s.coordinates * 1e-3, s.triangles)
    yield "screen32_large", M.Mesh(s.coordinates * 1e3, s.triangles)
    yield "graded", M.screen_graded(4, 8, 3.0)


@pytest.mark.parametrize("name,m", list(_meshes()))
def test_skipped_instants_have_no_front(oracle, name, m):
    cP, cS = 3 ** 0.5, 1.0
    rng = np.random.default_rng(11)
    scale = float(np.ptp(m.coordinates, axis=0).max())
    skipped = 0
    for trial in range(300):
        j = int(rng.integers(0, m.numberTriangles))
        T = m.coordinates[m.triangles[j]]
        ctr = T.mean(0)
        kind = trial % 3
        if kind == 0:        # off the plane, away from the triangle (beyond the absolute tolerances too)
            d = rng.normal(size=3)
            x = ctr + d / np.linalg.norm(d) * (scale * rng.uniform(0.1, 0.6) + rng.uniform(0.0, 0.05))
        elif kind == 1:      # near a vertex of another triangle of the mesh
            v = m.coordinates[int(rng.integers(0, m.number_nodes))]
            x = v + rng.normal(size=3) * scale * 1e-7
        else:                # in the triangle's plane, beyond an edge
            n = np.cross(T[1] - T[0], T[2] - T[0])
            n /= np.linalg.norm(n)
            d = rng.normal(size=3)
            d -= (d @ n) * n
            x = ctr + d / np.linalg.norm(d) * scale * rng.uniform(0.05, 0.6)
        b = reach(T, x)
        if not b > 0:
            continue
        for tau in (b / cP * (1 - 1e-12), b / cP * rng.uniform(0.0, 1.0)):
            if not cP * tau < b:
                continue
            _, typ = oracle.field_integrals(m, cP, cS, j, x, float(tau))
            assert typ == 0, (name, j, x, tau, b)
            skipped += 1
    assert skipped > 50
