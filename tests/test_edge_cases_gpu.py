"""Edge cases of the assembly and marching on the device: a one-triangle
mesh, lag windows past L, a single time step, a sliver
triangle (the thin-child case whose reference formulas amplify rounding),
against the binary128 oracle; and the C ABI's answers to invalid arguments."""
import ctypes as C

import numpy as np
import pytest

from conftest import cuda_available

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ebem():
    if not cuda_available():
        pytest.skip("no CUDA device")
    import elastodynamicebem_b200.core as core
    return core


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def test_single_triangle(ebem, oracle):
    from elastodynamicebem_b200 import mesh, problem
    m = mesh.Mesh(np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.2, 0.9, 0.0]]), np.array([[0, 1, 2]]))
    prm = problem.ProblemParams(1.0, 1.0, 2.0, 1.0, 10)
    dm = ebem.DeviceMesh(m)
    L = ebem.num_blocks(dm, prm)
    assert L == oracle.num_blocks(m, prm)
    E = ebem.assemble_sa(dm, prm, 7, 0, L).cpu().numpy()
    Eq, _ = oracle.assemble_sa(m, prm, 7, 0, L, variant="q")
    assert rel(E, Eq) <= 1e-10


def test_lags_past_the_last_non_null(ebem, oracle):
    from elastodynamicebem_b200 import mesh, problem
    m, prm = mesh.screen_uniform(2), problem.ProblemParams(1.0, 1.0, 2.0, 4.0, 40)   # dt = 0.1
    dm = ebem.DeviceMesh(m)
    L = ebem.num_blocks(dm, prm)
    assert L < prm.nT
    # the null test (centroid distance plus both longest edges) is more
    # generous than L (largest vertex distance), so blocks past L are assembled,
    # and are zero: every node pair is past both fronts, the second difference
    # of a constant
    E, cnt = ebem.assemble_sa(dm, prm, 7, L, 5, count=True)
    Eo, cnt_o = oracle.assemble_sa(m, prm, 7, L, 5)
    scale = float(ebem.assemble_sa(dm, prm, 7, 0, 1).abs().max())
    assert cnt == cnt_o
    assert float(E.abs().max()) <= 1e-13 * scale and np.abs(Eo).max() <= 1e-13 * scale


def test_single_time_step(ebem, oracle):
    from elastodynamicebem_b200 import mesh, problem
    m, prm = mesh.screen_uniform(2), problem.ProblemParams(1.0, 1.0, 2.0, 0.05, 1)
    dm = ebem.DeviceMesh(m)
    phi, L = ebem.timemarch_sa(dm, prm, 7, problem.DATUM_SCREEN_T4EXP)
    assert L == 1 and phi.shape == (1, 3 * m.numberTriangles)
    Eo, _ = oracle.assemble_sa(m, prm, 7, 0, 1)
    phio = oracle.march(Eo, oracle.rhs(m, prm, 7, problem.DATUM_SCREEN_T4EXP))
    assert rel(phi.cpu().numpy().T, phio) <= 1e-10


def test_sliver_triangle(ebem, oracle):
    """A triangle of aspect ratio 1e-3 beside a regular one: the children of
    its outer nodes are thin, where the reference's law-of-cosines form loses
    digits; the device form stays within 1e-10 of the binary128 value."""
    from elastodynamicebem_b200 import mesh, problem
    coords = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.5, 0.001, 0.0], [0.3, -0.8, 0.05]])
    m = mesh.Mesh(coords, np.array([[0, 1, 2], [1, 0, 3]]))
    prm = problem.ProblemParams(1.0, 1.0, 2.0, 1.0, 20)
    dm = ebem.DeviceMesh(m)
    L = ebem.num_blocks(dm, prm)
    E = ebem.assemble_sa(dm, prm, 7, 0, L).cpu().numpy()
    Eq, _ = oracle.assemble_sa(m, prm, 7, 0, L, variant="q")
    Eo, _ = oracle.assemble_sa(m, prm, 7, 0, L)
    assert rel(E, Eq) <= 1e-10
    print(f"\nsliver: device vs binary128 {rel(E, Eq):.1e}, FP64 restatement vs binary128 {rel(Eo, Eq):.1e}")


def test_invalid_arguments(ebem):
    import torch
    from elastodynamicebem_b200 import lib, mesh, problem
    L_ = lib.load()
    m, prm = mesh.screen_uniform(2), problem.ProblemParams(1.0, 1.0, 2.0, 1.0, 10)
    dm = ebem.DeviceMesh(m)
    p = lib.problem_struct(prm)
    n3 = 3 * m.numberTriangles
    out = torch.empty((4, n3, n3), dtype=torch.float64, device="cuda")
    ok = L_.ebem_assemble_sa(dm.handle, C.byref(p), 7, 0, 4, out.data_ptr(), 0, None, None)
    assert ok == 0
    assert L_.ebem_assemble_sa(dm.handle, C.byref(p), 7, 0, 0, out.data_ptr(), 0, None, None) == -1   # nlag < 1
    assert L_.ebem_assemble_sa(dm.handle, C.byref(p), 7, -1, 4, out.data_ptr(), 0, None, None) == -1  # lag0 < 0
    assert L_.ebem_assemble_sa(dm.handle, C.byref(p), 5, 0, 4, out.data_ptr(), 0, None, None) == -1   # no 5-node rule
    assert L_.ebem_assemble_sa(dm.handle, C.byref(p), 7, 0, 4, None, 0, None, None) == -1              # no output
    bad = lib.problem_struct(problem.ProblemParams(-1.0, 1.0, 2.0, 1.0, 10))
    assert L_.ebem_assemble_sa(dm.handle, C.byref(bad), 7, 0, 4, out.data_ptr(), 0, None, None) == -1  # rho <= 0
    assert L_.ebem_last_error()
    # post-processing times past tfin: the density has no column for them
    phi0 = torch.zeros((prm.nT, n3), dtype=torch.float64, device="cuda")
    pts = np.array([[0.1, 0.2, 0.3]])
    with pytest.raises(lib.EbemError):
        ebem.pp_sa(dm, prm, phi0, pts, np.array([0.5, prm.Tfin * 1.01]))
    with pytest.raises(lib.EbemError):
        ebem.pp_sa(dm, prm, phi0, pts, np.array([float("nan")]))
    u = ebem.pp_sa(dm, prm, phi0, pts, np.array([-1.0, prm.Tfin]))
    assert float(u.abs().max()) == 0.0
    # a zero E_0 cannot be factorised
    E = torch.zeros((2, n3, n3), dtype=torch.float64, device="cuda")
    b = torch.ones((3, n3), dtype=torch.float64, device="cuda")
    phi = torch.empty_like(b)
    assert L_.ebem_march(E.data_ptr(), n3, 2, b.data_ptr(), 3, phi.data_ptr(), None) == -5
