"""Right-hand side, time marching and post-processing on the device (through
the C ABI) against the oracle.

The density and displacement are judged like the blocks: against the
binary128 evaluation of the reference's formulas where affordable, with the
bar "no farther from it than the FP64 restatement of the reference", and
against the FP64 restatement within its own noise.
"""
import numpy as np
import pytest

from conftest import cuda_available

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.fixture(scope="module")
def ebem():
    if not cuda_available():
        pytest.skip("no CUDA device")
    import elastodynamicebem_b200.core as core
    return core


@pytest.mark.parametrize("datum", list(range(8)))
def test_rhs_matches_oracle(ebem, oracle, datum):
    from elastodynamicebem_b200 import mesh, problem
    for m, prm in [(mesh.screen_uniform(4), problem.ProblemParams(1, 1, 2, 1, 20)),
                   (mesh.icosphere(1), problem.ProblemParams(1, 1, 1, 2, 16))]:
        dm = ebem.DeviceMesh(m)
        b = ebem.rhs(dm, prm, 7, datum).cpu().numpy().T          # (3N, nT)
        bo = oracle.rhs(m, prm, 7, datum)
        if np.linalg.norm(bo) == 0:
            assert np.linalg.norm(b) == 0
        else:
            assert rel(b, bo) <= 1e-13


def test_march_matches_oracle(ebem, oracle):
    """Same blocks and right-hand side: device LU + history product vs the
    oracle's LU marching."""
    import torch
    from elastodynamicebem_b200 import mesh, problem
    m, prm = mesh.icosphere(1), problem.ProblemParams(1, 1, 1, 1, 40)
    L = oracle.num_blocks(m, prm)
    Eo, _ = oracle.assemble_sa(m, prm, 7, 0, L)
    bo = oracle.rhs(m, prm, 7, 1)
    phi_o = oracle.march(Eo, bo)
    E = torch.tensor(Eo, device="cuda")
    b = torch.tensor(bo.T.copy(), device="cuda")
    phi = ebem.march(E, b).cpu().numpy().T
    assert rel(phi, phi_o) <= 1e-11
    # host buffers through the same entry point
    phi_h = ebem.march(torch.tensor(Eo), torch.tensor(bo.T.copy())).numpy().T
    assert rel(phi_h, phi_o) <= 1e-11


def test_timemarch_screen128(ebem, oracle):
    """The screen workload end to end: 128 triangles, dt = 0.05, 20 steps,
    GH7, g = (0,0,t^4 e^{-2t})."""
    from elastodynamicebem_b200 import problem
    w = problem.screen_workload()
    m, prm = w.mesh, w.params
    dm = ebem.DeviceMesh(m)
    phi, L = ebem.timemarch_sa(dm, prm, 7, w.datum)
    phi = phi.cpu().numpy().T
    Eo, _ = oracle.assemble_sa(m, prm, 7, 0, L)
    bo = oracle.rhs(m, prm, 7, w.datum)
    phi_o = oracle.march(Eo, bo)
    assert np.isfinite(phi).all()
    assert rel(phi, phi_o) <= 1e-6          # FP64 restatement's own noise on this mesh: ~2e-8 in E


def test_timemarch_vs_exact_small(ebem, oracle):
    """Density from the device vs the density from the binary128 blocks."""
    from elastodynamicebem_b200 import mesh, problem
    m, prm = mesh.screen_uniform(4), problem.ProblemParams(1, 1, 2, 1, 20)
    dm = ebem.DeviceMesh(m)
    phi, L = ebem.timemarch_sa(dm, prm, 7, 0)
    phi = phi.cpu().numpy().T
    bo = oracle.rhs(m, prm, 7, 0)
    Eq, _ = oracle.assemble_sa(m, prm, 7, 0, L, variant="q")
    Ef, _ = oracle.assemble_sa(m, prm, 7, 0, L)
    phi_q = oracle.march(Eq, bo)
    phi_f = oracle.march(Ef, bo)
    e_dev, e_ref = rel(phi, phi_q), rel(phi_f, phi_q)
    assert e_dev <= max(1e-10, 3 * e_ref), (e_dev, e_ref)


def test_pp_screen(ebem, oracle):
    """Displacement on z = 0.3 from the device density; oracle evaluates the
    same closed form from the same density."""
    import torch
    from elastodynamicebem_b200 import problem
    w = problem.screen_workload()
    m, prm = w.mesh, w.params
    dm = ebem.DeviceMesh(m)
    phi, L = ebem.timemarch_sa(dm, prm, 7, w.datum)
    pts, times = w.points[:24], w.times[::3]
    u = ebem.pp_sa(dm, prm, phi, pts, times).cpu().numpy()          # (nt, np, 3)
    uo = oracle.pp_sa(m, prm, phi.cpu().numpy().T, pts, times)      # (3, np, nt)
    uo = uo.transpose(2, 1, 0)
    assert np.isfinite(u).all()
    assert rel(u, uo) <= 1e-9
    # exact value of the formulas at a few points and times
    uq = oracle.pp_sa(m, prm, phi.cpu().numpy().T, pts[:3], times[:2], variant="q").transpose(2, 1, 0)
    assert rel(u[:2, :3], uq) <= 1e-10


def test_pp_grid_and_off_grid_times(ebem, oracle):
    """Output times whose instants t - k dt repeat (on the grid, or all with
    one offset from it) take the path that evaluates each distinct instant
    once per (triangle, point); scattered times the per-time path; t <= 0
    gives zero.  All against the oracle's closed form."""
    from elastodynamicebem_b200 import problem
    w = problem.screen_workload()
    m, prm = w.mesh, w.params
    dm = ebem.DeviceMesh(m)
    phi, L = ebem.timemarch_sa(dm, prm, 7, w.datum)
    pts = w.points[:16]
    # within the simulated interval: past t = (nT - 1) dt the reference's sum
    # reads density columns that do not exist (BEMenerg_postProcA_singlePoint.m:21,58)
    on = np.concatenate([[0.0], prm.dt * np.array([1, 2, 7, 13, prm.nT - 1])])
    offset = np.concatenate([[0.0], prm.dt * (np.array([0, 1, 6, 12, prm.nT - 2]) + 0.37)])
    scattered = np.concatenate([[-0.1], np.random.default_rng(4).uniform(0.0, (prm.nT - 1) * prm.dt, 6)])
    for times in (on, offset, scattered):
        u = ebem.pp_sa(dm, prm, phi, pts, times).cpu().numpy()
        uo = oracle.pp_sa(m, prm, phi.cpu().numpy().T, pts, times).transpose(2, 1, 0)
        assert np.abs(u[0]).max() == 0.0 if times[0] == 0.0 else True
        assert rel(u, uo) <= 1e-9


def test_pp_sphere1280_point_chunks(ebem, oracle):
    """The benchmark sphere's 256 exterior points at its 40 grid times: the
    instant path runs in two chunks of points (its buffer is capped at
    1 GiB: 151 points of 1280 triangles x 115 instants), and 97 % of the
    (triangle, point, instant) items lie before the P front and are skipped.
    Points on both sides of the chunk boundary against the oracle."""
    from elastodynamicebem_b200 import problem
    w = problem.sphere_workload(7)
    dm = ebem.DeviceMesh(w.mesh)
    phi, L = ebem.timemarch_sa(dm, w.params, 7, w.datum)
    u = ebem.pp_sa(dm, w.params, phi, w.points, w.times).cpu().numpy()          # (times, points, 3)
    sel = [0, 77, 150, 151, 152, 255]
    uo = oracle.pp_sa(w.mesh, w.params, phi.cpu().numpy().T, w.points[sel], w.times).transpose(2, 1, 0)
    assert np.isfinite(u).all()
    assert rel(u[:, sel], uo) <= 1e-9


def test_workspace_pool_reuse_and_release(ebem, oracle):
    """Per-call workspaces come from the library's stream-ordered pool: repeated
    calls reuse it, ebem_release_workspace hands it back, and calls after the
    release allocate again; every call gives the same displacement (to
    rounding: the per-time path adds with atomics)."""
    from elastodynamicebem_b200 import lib, problem
    w = problem.screen_workload()
    dm = ebem.DeviceMesh(w.mesh)
    phi, L = ebem.timemarch_sa(dm, w.params, 7, w.datum)
    pts, times = w.points[:16], w.times
    u1 = ebem.pp_sa(dm, w.params, phi, pts, times).cpu().numpy()
    u2 = ebem.pp_sa(dm, w.params, phi, pts, times).cpu().numpy()
    lib.check(lib.load().ebem_release_workspace())
    u3 = ebem.pp_sa(dm, w.params, phi, pts, times).cpu().numpy()
    # the history product adds with atomics: equal to rounding, not bitwise
    assert rel(u2, u1) <= 1e-13 and rel(u3, u1) <= 1e-13
    phi2, _ = ebem.timemarch_sa(dm, w.params, 7, w.datum)
    assert rel(phi2.cpu().numpy(), phi.cpu().numpy()) <= 1e-13


def test_cholesky_of_symmetric_part(ebem, oracle):
    """A Cholesky factorisation of E_0 beside the LU: it factors the
    symmetric part (E_0 + E_0^T) / 2 (E_0 of the outer-quadrature /
    exact-inner assembly is not symmetric: 8.0e-3 relative on this mesh), and
    the marching with it equals a float64 numpy marching with that symmetric
    part to 1e-12; against the reference's LU marching the density differs by
    the asymmetry's effect, measured here and bounded."""
    import torch
    from elastodynamicebem_b200 import problem
    w = problem.screen_workload()
    dm = ebem.DeviceMesh(w.mesh)
    L = ebem.num_blocks(dm, w.params)
    E = ebem.assemble_sa(dm, w.params, 7, 0, L)
    b = ebem.rhs(dm, w.params, 7, w.datum)
    phi_lu = ebem.march(E, b).cpu().numpy()
    phi_ch = ebem.march(E, b, factor=ebem.FACTOR_CHOLESKY).cpu().numpy()
    En, bn = E.cpu().numpy(), b.cpu().numpy()
    E0 = En[0]
    asym = np.linalg.norm(E0 - E0.T) / np.linalg.norm(E0)
    assert 5e-3 < asym < 1.2e-2
    S = 0.5 * (E0 + E0.T)
    ref = np.zeros_like(bn)
    for n in range(bn.shape[0]):
        rhs_n = bn[n].copy()
        for l in range(1, min(n + 1, L)):
            rhs_n -= En[l] @ ref[n - l]
        ref[n] = np.linalg.solve(S, rhs_n)
    assert rel(phi_ch, ref) <= 1e-12
    d = rel(phi_ch, phi_lu)
    print(f"E_0 asymmetry {asym:.2e}; density Cholesky(sym part) vs LU {d:.2e}")
    assert d < 0.1


def test_cholesky_rejects_indefinite(ebem):
    import torch
    from elastodynamicebem_b200.lib import EbemError
    A = -torch.eye(6, dtype=torch.float64, device="cuda").unsqueeze(0)
    b = torch.ones((2, 6), dtype=torch.float64, device="cuda")
    with pytest.raises(EbemError) as ei:
        ebem.march(A, b, factor=ebem.FACTOR_CHOLESKY)
    assert ei.value.code == -5 and "positive definite" in str(ei.value)
    assert torch.allclose(ebem.march(A, b), -b)                   # LU of the same matrix is fine
