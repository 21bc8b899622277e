"""Numerical post-processing of the indirect formulation (the reference's
method "GPU yy z") on the device, through the C ABI (ebem_pp_gpu), against:

* the reference's own kernels, kernelSP and kernelLayer, compiled from its
  sources into oracle/_ref and run on the same GPU (kernelSP's matrix summed
  on the host as BEMenerg_postProcGPU_calcSP.m:78-85 does; kernelLayer
  contracts in the kernel), bar 1e-12;
* the oracle's C++ restatement of both (oracle.pp_gpu), bar 1e-12;
* the closed-form post-processing (ebem_pp_sa): the numerical result
  converges to it as the composite rule refines.

The reference's node-stride defect (kernelSP.cu:41 reads node 3 * subregion
+ l) is reproduced by default and fixed with EBEM_FIX_REFERENCE_DEFECTS.
"""
import numpy as np
import pytest

from conftest import cuda_available

pytestmark = pytest.mark.gpu

TOL = 1e-12


def rel(a, b):
    """Relative Frobenius difference; the absolute one where b is zero (before
    the P front reaches any point both are exactly zero)."""
    a, b = np.asarray(a), np.asarray(b)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / nb) if nb > 0 else float(np.linalg.norm(a))


@pytest.fixture(scope="module")
def ebem():
    if not cuda_available():
        pytest.skip("no CUDA device")
    import elastodynamicebem_b200.core as core
    return core


@pytest.fixture(scope="module")
def screen(ebem):
    """Screen of 32 triangles marched over 20 steps; points above it (z =
    0.31, off the height 6 c_S dt where a front radius equals the height),
    times on and off the time grid."""
    from elastodynamicebem_b200 import mesh, problem
    m, prm = mesh.screen_uniform(4), problem.ProblemParams(1.0, 1.0, 2.0, 1.0, 20)
    dm = ebem.DeviceMesh(m)
    phi, _ = ebem.timemarch_sa(dm, prm, 7, 0)
    rng = np.random.default_rng(21)
    pts = np.column_stack([rng.uniform(-0.5, 0.5, 12), rng.uniform(-0.5, 0.5, 12), np.full(12, 0.31)])
    times = np.concatenate([prm.dt * np.array([1, 4, 9, 15, 19]), [0.377, 0.0, -0.2]])
    return m, prm, dm, phi, pts, times


@pytest.mark.parametrize("variant", [0, 1])
@pytest.mark.parametrize("n_sub,n_sing", [(1, 3), (4, 3), (16, 3), (4, 7), (16, 19), (64, 1), (1, 12)])
def test_matches_restatement(ebem, oracle, screen, variant, n_sub, n_sing):
    m, prm, dm, phi, pts, times = screen
    stride = n_sing if variant == 1 else 3
    if variant == 0 and (n_sub - 1) * 3 + n_sing > n_sub * n_sing:
        pytest.skip("kernelSP's stride-3 read passes the node table for this rule (tested below)")
    u = ebem.pp_gpu(dm, prm, phi, pts, times, n_sub, n_sing, variant).cpu().numpy().transpose(2, 1, 0)
    uo = oracle.pp_gpu(m, prm, phi.cpu().numpy().T, pts, times, n_sub, n_sing, variant, stride)
    assert np.isfinite(u).all()
    assert np.abs(u[:, :, times <= 0]).max() == 0.0
    assert rel(u, uo) <= TOL


def test_stride_defect_flag(ebem, oracle, screen):
    """kernelSP's stride-3 node read changes the 7-node rule's result; the fix
    flag reads the rule's own nodes (then both variants agree to rounding and
    the clean-up thresholds); rules whose stride-3 read would pass the end of
    the table are refused unless the flag is given."""
    from elastodynamicebem_b200.lib import EbemError
    m, prm, dm, phi, pts, times = screen
    ref = ebem.pp_gpu(dm, prm, phi, pts, times, 4, 7, 0).cpu().numpy()
    fixed = ebem.pp_gpu(dm, prm, phi, pts, times, 4, 7, 0, fix_defects=True).cpu().numpy()
    layer = ebem.pp_gpu(dm, prm, phi, pts, times, 4, 7, 1).cpu().numpy()
    assert rel(fixed, ref) > 1e-4
    assert rel(fixed, layer) <= 1e-12
    uo = oracle.pp_gpu(m, prm, phi.cpu().numpy().T, pts, times, 4, 7, 0, 7)
    assert rel(fixed, uo.transpose(2, 1, 0)) <= TOL
    with pytest.raises(EbemError) as ei:
        ebem.pp_gpu(dm, prm, phi, pts, times, 4, 1, 0)
    assert ei.value.code == -1 and "kernelSP.cu:41" in str(ei.value)
    ok = ebem.pp_gpu(dm, prm, phi, pts, times, 4, 1, 0, fix_defects=True).cpu().numpy()
    assert np.isfinite(ok).all()


def test_converges_to_closed_form(ebem, screen):
    m, prm, dm, phi, pts, times = screen
    ua = ebem.pp_sa(dm, prm, phi, pts, times[:5]).cpu().numpy()
    errs = [rel(ebem.pp_gpu(dm, prm, phi, pts, times[:5], ns, 3, 1).cpu().numpy(), ua) for ns in (1, 4, 16, 64)]
    assert errs[-1] < errs[0] / 4 and errs[-1] < 1e-3, errs


def test_matches_reference_kernels(ebem, oracle, screen):
    if not oracle.ref_pp_available():
        pytest.skip("oracle/_ref kernelSP / kernelLayer not built (reference sources absent when building)")
    m, prm, dm, phi, pts, times = screen
    ph = phi.cpu().numpy().T
    for n_sub, n_sing in ((16, 3), (4, 7), (64, 3)):
        # kernelSP: one point, its times (u(x, :))
        x = pts[3]
        u = ebem.pp_gpu(dm, prm, phi, x[None], times, n_sub, n_sing, 0).cpu().numpy()[:, 0]      # (nt, 3)
        ur = np.stack([oracle.ref_pp_sp(m, prm, ph, x, t, n_sub, n_sing)[0] for t in times])
        assert rel(u, ur) <= TOL, (n_sub, n_sing)
        # kernelLayer: all points at one time (u(:, t))
        for t in times[:4]:
            ul = ebem.pp_gpu(dm, prm, phi, pts, [t], n_sub, n_sing, 1).cpu().numpy()[0].T        # (3, npts)
            ulr = oracle.ref_pp_layer(m, prm, ph, pts, t, n_sub, n_sing)[0]
            assert rel(ul, ulr) <= TOL, (n_sub, n_sing, t)


def test_bench_sizes(ebem, oracle):
    """The sphere benchmark's size: 1280 triangles, 40 steps, 256 exterior
    points at all 40 times, composite rule 16 x 3; sampled against the
    restatement, every output finite."""
    from elastodynamicebem_b200 import problem
    w = problem.sphere_workload(7)
    dm = ebem.DeviceMesh(w.mesh)
    phi, _ = ebem.timemarch_sa(dm, w.params, 7, w.datum)
    u = ebem.pp_gpu(dm, w.params, phi, w.points, w.times, 16, 3, 1).cpu().numpy()
    assert u.shape == (40, 256, 3) and np.isfinite(u).all()
    sel = np.array([0, 77, 200])
    uo = oracle.pp_gpu(w.mesh, w.params, phi.cpu().numpy().T, w.points[sel], w.times[[9, 39]], 16, 3, 1)
    assert rel(u[[9, 39]][:, sel].transpose(2, 1, 0), uo) <= TOL
