"""Numerical-inner assembly (the reference's kernelGHC / kernelV path) on the
device against the oracle's restatement of kernelGHC.cu, and the diagonal
from the semi-analytic kernel (the reference's GPU method)."""
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


@pytest.mark.parametrize("n_gh,n_sub,n_sing", [(7, 16, 3), (12, 64, 3), (7, 16, 19), (3, 1, 7)])
def test_ghc_matches_oracle(ebem, oracle, n_gh, n_sub, n_sing):
    from elastodynamicebem_b200 import mesh, problem
    m, prm = mesh.icosphere(1), problem.ProblemParams(1, 1, 1, 1, 40)
    dm = ebem.DeviceMesh(m)
    L = ebem.num_blocks(dm, prm)
    E = ebem.assemble_ghc(dm, prm, n_gh, n_sub, n_sing, 0, L, sa_diagonal=False).cpu().numpy()
    Eo = oracle.assemble_ghc(m, prm, n_gh, n_sub, n_sing, 0, L)
    assert np.isfinite(E).all()
    assert rel(E, Eo) <= 1e-10
    for l in range(0, L, 7):
        if np.linalg.norm(Eo[l]) > 0:
            assert rel(E[l], Eo[l]) <= 1e-9


def test_gpu_method_diagonal_is_sa(ebem):
    from elastodynamicebem_b200 import mesh, problem
    m, prm = mesh.screen_uniform(4), problem.ProblemParams(1, 1, 2, 1, 20)
    dm = ebem.DeviceMesh(m)
    L = ebem.num_blocks(dm, prm)
    E = ebem.assemble_ghc(dm, prm, 7, 16, 3, 0, L, sa_diagonal=True).cpu().numpy()
    S = ebem.assemble_sa(dm, prm, 7, 0, L).cpu().numpy()
    N = m.numberTriangles
    # the diagonal blocks come from the diagonal-only semi-analytic kernel:
    # equal to the full assembly's to rounding (the same terms in another order)
    for i in range(N):
        d, s = E[:, 3 * i:3 * i + 3, 3 * i:3 * i + 3], S[:, 3 * i:3 * i + 3, 3 * i:3 * i + 3]
        assert np.abs(d - s).max() <= 1e-14 * np.abs(s).max()
    # off-diagonal numerical blocks approach the semi-analytic ones as the inner rule refines
    mask = np.ones((3 * N, 3 * N), bool)
    for i in range(N):
        mask[3 * i:3 * i + 3, 3 * i:3 * i + 3] = False
    coarse = rel(E[:, mask], S[:, mask])
    fine = rel(ebem.assemble_ghc(dm, prm, 7, 64, 19, 0, L, sa_diagonal=True).cpu().numpy()[:, mask], S[:, mask])
    assert fine < coarse


def test_reference_kernel_pins_restatement(ebem, oracle):
    """The reference's own kernelGHC.cu, compiled from its source into
    oracle/_ref and run on the device, against the oracle's CPU restatement
    of it and against the device numerical-inner kernel."""
    if not oracle.ref_ghc_available():
        pytest.skip("oracle/_ref/libref_ghc.so not built (reference sources absent when building)")
    from elastodynamicebem_b200 import mesh, problem
    m, prm = mesh.icosphere(1), problem.ProblemParams(1, 1, 1, 1, 40)
    L = oracle.num_blocks(m, prm)
    Er = oracle.ref_ghc(m, prm, 7, 16, 3, L)
    Eo = oracle.assemble_ghc(m, prm, 7, 16, 3, 0, L)
    dm = ebem.DeviceMesh(m)
    Ed = ebem.assemble_ghc(dm, prm, 7, 16, 3, 0, L, sa_diagonal=False).cpu().numpy()
    assert rel(Eo, Er) <= 1e-12, "oracle restatement vs the reference's kernel"
    assert rel(Ed, Er) <= 1e-10, "device kernel vs the reference's kernel"
