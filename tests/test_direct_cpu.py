"""Direct-formulation oracle and data on the CPU: the DIAG rule, the P1 basis,
the bar data of the reference and basic structure of the restated operators."""
import numpy as np
import pytest


@pytest.mark.parametrize("n", [16, 64, 256])
def test_diag_rule_exact(oracle, n):
    """doppioGauss1D: collapsed Gauss-Legendre, exact for low-degree
    polynomials in the barycentric coordinates (area-normalised)."""
    nodes, w = oracle.doppio_gauss(n)
    assert abs(w.sum() - 1) < 1e-14
    assert np.abs(nodes.sum(1) - 1).max() < 1e-15
    # int l_a^p l_b^q l_c^r dA / A = 2 p! q! r! / (p+q+r+2)!
    from math import factorial
    for p, q, r in [(1, 0, 0), (0, 0, 2), (1, 1, 0), (2, 1, 1), (0, 3, 1)]:
        exact = 2 * factorial(p) * factorial(q) * factorial(r) / factorial(p + q + r + 2)
        got = (w * nodes[:, 0] ** p * nodes[:, 1] ** q * nodes[:, 2] ** r).sum()
        assert abs(got - exact) < 1e-14


def test_diag_rule_rejects_non_square(oracle):
    with pytest.raises(ValueError):
        oracle.doppio_gauss(20)


def test_p1_basis(oracle):
    from elastodynamicebem_b200 import mesh
    m = mesh.prism_bar(1.0, 1.0, 3.0, 0.5)
    for unit in (False, True):
        M, v = oracle.p1_coeffs(m, unit)
        for t in range(0, m.numberTriangles, 7):
            V = m.coordinates[m.triangles[t]]
            phi = v[t][:, None] + M[t] @ V.T
            assert np.abs(phi - np.eye(3)).max() < 1e-12


def test_bar_data():
    """Closed forms of the 1-D bar (height h): before the first reflection the
    top face (x3 = h, n3 = 1) carries traction 2 mu, the displacement there is
    c_P t, and the lateral faces carry no traction."""
    from elastodynamicebem_b200 import mesh, problem
    m = mesh.prism_bar(1.0, 1.0, 3.0, 0.5)
    prm = problem.ProblemParams(1.0, 1.0, 2.0, 2.0, 20)
    gV = problem.bar_neumann(m, prm, 3.0)
    gK = problem.bar_dirichlet(m, prm, 3.0)
    top = np.where(np.abs(m.center[:, 2] - 3.0) < 1e-12)[0]
    side = np.where(np.abs(m.normal[:, 2]) < 1e-12)[0]
    assert len(top) and len(side)
    n = 3                                    # t = 0.3, c_P t = 0.6 < 2 h
    assert np.allclose(gV[n - 1, 3 * top + 2], 2 * prm.mu)
    assert np.all(gV[:, 3 * side + 2] == 0) and np.all(gV[:, 0::3] == 0)
    vt = np.where(np.abs(m.coordinates[:, 2] - 3.0) < 1e-12)[0]
    assert np.allclose(gK[n - 1, 3 * vt + 2], prm.velP * n * prm.dt)


def test_oracle_k_structure(oracle):
    """K_l vanishes beyond L_K; the singular part lives on the (triangle,
    own vertex) blocks only and is zero after ceil(maxL / (c_S dt)) + 2 lags."""
    from elastodynamicebem_b200 import mesh, problem
    m = mesh.prism_bar(1.0, 1.0, 3.0, 1.0)
    prm = problem.ProblemParams(1.0, 1.0, 2.0, 2.0, 10)
    LV, LK = oracle.num_blocks_dir(m, prm)
    Ks = oracle.k_sing(m, prm, 3, 16, 0, LK)
    mask = np.zeros((3 * m.numberTriangles, 3 * m.number_nodes), bool)
    for x, tri in enumerate(m.triangles):
        for s in tri:
            mask[3 * x:3 * x + 3, 3 * s:3 * s + 3] = True
    assert np.all(Ks[:, ~mask] == 0)
    lmax = int(np.ceil(m.maxL.max() / (prm.velS * prm.dt))) + 2
    if lmax < LK:
        assert np.all(Ks[lmax:] == 0)
    assert np.abs(Ks[0]).max() > 0
    K = oracle.assemble_k(m, prm, 3, 1, 3, 0, LK + 2, nblocks=LK)
    assert np.all(K[LK:] == 0) and np.isfinite(K).all()
