"""The semi-analytic assembly pinned to code the reference itself runs, and
to the exact value of the reference's formulas at the benchmark sizes.

1. Against the reference's own kernelGHC (kernelGHC.cu:5-167, compiled from
   its source file into oracle/_ref and run on the device).  kernelGHC
   evaluates the same E_l blocks with the same outer Gauss-Hammer rule but a
   numerical inner rule (composite Gauss-Hammer on n_sub sub-triangles); the
   semi-analytic method (BEMenerg_coreSA_calcMatrixSubBlock.m:1-111) takes
   the inner integral in closed form.  As the inner rule refines, kernelGHC's
   blocks must converge to the device's semi-analytic blocks at the rate of
   the composite rule on this integrand: the Lame kernel jumps across the
   wavefronts (the H(t - r/c) factors of kernelGHC.cu:204-259) and is
   singular at shared edges, so the error falls like the sub-triangle size h,
   halving with each fourfold refinement.  Rules with more nodes than the
   kernel's 1024-thread block holds run as chunks of sub-triangles
   (oracle.ref_ghc_composite).
2. Against binary128 fixtures (tests/golden/make_golden_bench.py) at the
   benchmark configurations: sampled blocks of the 1280-triangle sphere with
   the 7- and 12-node rules, and the screen benchmark's time-marched density
   (all 20 steps) and post-processed displacement at all 100 points x 20
   times.  Bar: 1e-10 relative.
"""
import os

import numpy as np
import pytest

from conftest import ROOT, cuda_available

pytestmark = pytest.mark.gpu

TOL = 1e-10
GOLDEN = os.path.join(ROOT, "tests", "golden", "bench_configs.npz")


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.fixture(scope="module")
def ebem():
    if not cuda_available():
        pytest.skip("no CUDA device")
    import elastodynamicebem_b200.core as core
    return core


def _patch(m, seed, n_near=24, n_far=24):
    """Triangles of one neighbourhood (adjacent and near pairs) plus scattered
    ones (well-separated pairs), as a mesh of their own."""
    from elastodynamicebem_b200 import mesh
    rng = np.random.default_rng(seed)
    c = m.center
    p = c[rng.integers(len(c))]
    near = np.argsort(np.linalg.norm(c - p, axis=1))[:n_near]
    far = rng.choice(np.setdiff1d(np.arange(len(c)), near), n_far, replace=False)
    return mesh.Mesh(m.coordinates, m.triangles[np.concatenate([near, far])])


@pytest.mark.parametrize("case", ["screen128", "sphere1280"])
@pytest.mark.parametrize("n_sing", [3, 19])
def test_converges_to_reference_kernel(ebem, oracle, case, n_sing):
    if not oracle.ref_ghc_available():
        pytest.skip("oracle/_ref/libref_ghc.so not built (reference sources absent when building)")
    from elastodynamicebem_b200 import problem
    w = problem.screen_workload() if case == "screen128" else problem.sphere_workload(7)
    L = oracle.num_blocks(w.mesh, w.params)
    m = _patch(w.mesh, 11 if case == "screen128" else 12)
    dm = ebem.DeviceMesh(m)
    sa = ebem.assemble_sa(dm, w.params, 7, 0, L).cpu().numpy()
    n3 = 3 * m.numberTriangles
    off = np.ones((n3, n3), bool)
    for i in range(m.numberTriangles):
        off[3 * i:3 * i + 3, 3 * i:3 * i + 3] = False          # kernelGHC skips the diagonal blocks
    errs = []
    for n_sub in (4, 16, 64, 256):
        g = oracle.ref_ghc_composite(m, w.params, 7, n_sub, n_sing, L)
        errs.append(rel(g[:, off], sa[:, off]))
    print(f"{case} n_sing={n_sing}: |SA - kernelGHC(n_sub)| / |SA| for n_sub = 4, 16, 64, 256: "
          + ", ".join(f"{e:.3e}" for e in errs))
    rates = [errs[k] / errs[k + 1] for k in range(3)]
    assert all(r > 1.3 for r in rates), rates                    # first order: about 2 per level
    assert errs[0] / errs[-1] > 4.0, errs
    assert errs[-1] < 0.05, errs


@pytest.fixture(scope="module")
def golden():
    if not os.path.exists(GOLDEN):
        pytest.skip("tests/golden/bench_configs.npz missing (python tests/golden/make_golden_bench.py)")
    return np.load(GOLDEN)


@pytest.mark.parametrize("n_gh", [7, 12])
def test_sphere1280_blocks_exact(ebem, golden, n_gh):
    """The headline workload (sphere of 1280 triangles, L = 40) assembled in
    full on the device; a seeded sample of 300 blocks against binary128."""
    from elastodynamicebem_b200 import problem
    w = problem.sphere_workload(n_gh)
    dm = ebem.DeviceMesh(w.mesh)
    L = ebem.num_blocks(dm, w.params)
    E = ebem.assemble_sa(dm, w.params, n_gh, 0, L)
    key = f"sphere1280_gh{n_gh}"
    src, fld, lag = golden[f"{key}/src"], golden[f"{key}/fld"], golden[f"{key}/lag"]
    exact, f64 = golden[f"{key}/exact"], golden[f"{key}/f64"]
    got = np.stack([E[l, 3 * i:3 * i + 3, 3 * j:3 * j + 3].cpu().numpy() for i, j, l in zip(src, fld, lag)])
    del E
    e_dev = rel(got, exact)
    print(f"{key}: device {e_dev:.2e}, FP64 restatement {rel(f64, exact):.2e} (vs binary128)")
    assert e_dev <= TOL
    assert np.abs(got - exact).max() <= TOL * np.abs(exact).max()


def test_screen128_density_and_displacement_exact(ebem, golden):
    """The screen benchmark end to end on the device (assembly, right-hand
    side, marching, closed-form post-processing at all 100 points x 20
    times) against the same chain in binary128."""
    from elastodynamicebem_b200 import problem
    w = problem.screen_workload()
    dm = ebem.DeviceMesh(w.mesh)
    phi, L = ebem.timemarch_sa(dm, w.params, w.n_gh, w.datum)
    u = ebem.pp_sa(dm, w.params, phi, w.points, w.times).cpu().numpy().transpose(2, 1, 0)    # (3, np, nt)
    phi = phi.cpu().numpy().T                                                                  # (3N, nT)
    phi_q, u_q = golden["screen128/phi_exact"], golden["screen128/u_exact"]
    e_phi, e_u = rel(phi, phi_q), rel(u, u_q)
    print(f"screen128 vs binary128: density {e_phi:.2e} (FP64 restatement "
          f"{rel(golden['screen128/phi_f64'], phi_q):.2e}), displacement {e_u:.2e} (FP64 restatement "
          f"{rel(golden['screen128/u_f64'], u_q):.2e})")
    assert u.shape == (3, 100, 20)
    assert e_phi <= TOL and e_u <= TOL
    # every step and every output time on its own
    for n in range(phi.shape[1]):
        if np.linalg.norm(phi_q[:, n]) > 0:
            assert rel(phi[:, n], phi_q[:, n]) <= TOL
    for q in range(u.shape[2]):
        if np.linalg.norm(u_q[:, :, q]) > 0:
            assert rel(u[:, :, q], u_q[:, :, q]) <= TOL
