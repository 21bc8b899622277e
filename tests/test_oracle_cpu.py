"""CPU checks of the oracle itself: it reproduces the committed golden
fixtures (FP64 and binary128 values of the reference's formulas), its
closed-form kernel integrals agree with an independent polar cubature, and
its null-test census matches the counts of non-null pair-lags (257,430 on
the generated 128-triangle screen, 257,204 on the reference's own
screenUniform_2 mesh)."""
import os
import sys

import numpy as np
import pytest

from conftest import ROOT

sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("case", ["screen32_gh7", "sphere80_gh12", "prism28_gh7", "limit32_gh7"])
def test_oracle_reproduces_golden(oracle, case):
    import make_golden
    z = np.load(os.path.join(ROOT, "tests", "golden", "sa_blocks.npz"))
    name, m, prm, n_gh = [c for c in make_golden.cases() if c[0] == case][0]
    src, fld, lag = z[f"{case}/src"], z[f"{case}/fld"], z[f"{case}/lag"]
    f = oracle.assemble_sa_pairs(m, prm, n_gh, src, fld, lag)
    q = oracle.assemble_sa_pairs(m, prm, n_gh, src, fld, lag, variant="q")
    assert rel(f, z[f"{case}/f64"]) <= 1e-15
    assert rel(q, z[f"{case}/exact"]) <= 1e-15


def test_closed_form_vs_polar_cubature(oracle):
    """ris1..ris6 of the closed form (binary128 evaluation) against an
    adaptive polar cubature that shares nothing with it.  The reference's
    formulas deliberately skip child triangles with doubled area below 1e-6
    and treat front/edge intersections with discriminant below 1e-6 as
    tangent (childTriangle.m:62,75; fieldTriangle.m:23), so they differ from
    the true integral by up to ~1e-6 relative in the configurations that
    trigger those thresholds; elsewhere the agreement is ~1e-13."""
    import polar_cubature as PC
    from elastodynamicebem_b200 import mesh
    m = mesh.icosphere(1)
    cP, cS = 3 ** 0.5, 1.0
    rng = np.random.default_rng(0)
    checked = 0
    errs = []
    for trial in range(40):
        j = int(rng.integers(0, m.numberTriangles))
        T = m.coordinates[m.triangles[j]]
        x = T.mean(0) + rng.normal(size=3) * 0.3
        t = float(rng.uniform(0.05, 0.8))
        ref, typ = oracle.field_integrals(m, cP, cS, j, x, t, variant="q")
        if typ == 0:
            continue
        pc = PC.kernel_integrals(T, x, t, cP, cS)
        e = max(np.abs(ref[k] - pc[k]).max() / np.abs(pc[k]).max() for k in range(6) if np.abs(pc[k]).max() > 0)
        errs.append(e)
        checked += 1
    assert checked >= 20
    errs = np.array(errs)
    assert np.max(errs) <= 1e-6
    assert np.mean(errs <= 1e-11) >= 0.8, errs


def test_null_census_screen():
    """Non-null pair-lags of the 8x8 screen problem (L = 20) with the
    reference's null test."""
    import oracle as O
    from elastodynamicebem_b200 import problem
    w = problem.screen_workload()
    L = O.num_blocks(w.mesh, w.params)
    assert L == 20
    assert O.count_nonnull(w.mesh, w.params, L) == 257430


def test_reference_mesh_census():
    """On the reference's own screenUniform_2 mesh the census is 257,204
    (runs only where the reference is mounted)."""
    from conftest import reference_file
    path = reference_file("mesh", "screenUniform", "screenUniform_2.mesh")
    import oracle as O
    from elastodynamicebem_b200 import mesh, problem
    m = mesh.read_space_mesh(path)
    prm = problem.ProblemParams(1.0, 1.0, 2.0, 1.0, 20)
    assert O.count_nonnull(m, prm, 20) == 257204


def test_sphere_census():
    """The benchmark's unit count: the generated icosphere of 1280 triangles
    (L = 40) has 26,678,800 non-null pair-lags; the reference's own
    sphereUniform_3 mesh, whose vertices lie elsewhere, has 26,137,900 (runs
    only where the reference is mounted)."""
    import oracle as O
    from elastodynamicebem_b200 import mesh, problem
    w = problem.sphere_workload(7)
    assert O.num_blocks(w.mesh, w.params) == 40
    assert O.count_nonnull(w.mesh, w.params, 40) == 26_678_800
    from conftest import REFERENCE_ROOT
    path = os.path.join(REFERENCE_ROOT, "mesh", "sphereUniform", "sphereUniform_3.mesh")
    if os.path.exists(path):
        assert O.count_nonnull(mesh.read_space_mesh(path), w.params, 40) == 26_137_900


def test_flop_census_frozen(oracle):
    """The frozen FP64 flops per pair-integral used by bench.py's roofline."""
    import importlib.util
    from elastodynamicebem_b200 import problem
    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    w = problem.sphere_workload(7)
    c = oracle.flop_census(w.mesh, w.params, 7, 1000, 0)
    assert abs(c["flops_per_pair_integral"] / bench.FLOPS_PER_PAIR_INTEGRAL - 1) < 0.03


def test_e0_asymmetry_and_definiteness():
    """E_0 of the semi-analytic assembly is not symmetric (the outer rule
    integrates the source triangle, the inner integral is exact on the field
    triangle): on the screen benchmark with the 7-node rule the relative
    asymmetry is 8.0e-3 and its symmetric part is positive definite, the two
    facts behind offering both LU (the reference's) and the Cholesky of the
    symmetric part."""
    import oracle as O
    from elastodynamicebem_b200 import problem
    w = problem.screen_workload()
    E, _ = O.assemble_sa(w.mesh, w.params, 7, 0, 1)
    E0 = E[0]
    asym = np.linalg.norm(E0 - E0.T) / np.linalg.norm(E0)
    assert abs(asym - 7.96e-3) < 2e-4
    ev = np.linalg.eigvalsh(0.5 * (E0 + E0.T))
    assert ev.min() > 0 and ev.max() / ev.min() < 10
