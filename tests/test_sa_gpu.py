"""Parity of the CUDA semi-analytic assembly (through the C ABI) with the CPU
oracle (C++ restatement of the reference's SA path).

Two oracles check the device result on the same double inputs:
  * "q"   the reference's formulas evaluated in binary128 (the exact value of
          those formulas to ~1e-30);
  * "f64" the same restatement in double precision, i.e. the reference's own
          arithmetic, whose rounding noise on these formulas reaches 1e-8
          relative on structured meshes (thin child triangles make the skew
          B-basis of coeffB.m amplify rounding by 1/sin^2(gamma)).
Bar: relative error <= 1e-10 against the exact value (the device evaluates
the same integrals in a stable form and lands near 1e-14), and within 1e-7 of
the FP64 restatement (its own noise).
"""
import numpy as np
import pytest

from conftest import cuda_available

pytestmark = pytest.mark.gpu

TOL = 1e-10          # relative Frobenius error where the reference's FP64 evaluation is itself that accurate
NOISE = 3.0          # allowed multiple of the FP64 restatement's own distance to the exact value
TOL_F64 = 1e-7       # device vs the FP64 restatement, relative Frobenius over all lags


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / nb if nb > 0 else np.linalg.norm(a)


@pytest.fixture(scope="module")
def ebem():
    if not cuda_available():
        pytest.skip("no CUDA device")
    import elastodynamicebem_b200.core as core
    return core


def _case(name):
    from elastodynamicebem_b200 import mesh, problem
    P = problem.ProblemParams
    if name == "screen32":
        return mesh.screen_uniform(4), P(1.0, 1.0, 2.0, 1.0, 20)
    if name == "screen128":
        return mesh.screen_uniform(8), P(1.0, 1.0, 2.0, 1.0, 20)
    if name == "sphere80":
        return mesh.icosphere(1), P(1.0, 1.0, 1.0, 1.0, 40)
    if name == "prism":      # source nodes at distance exactly c_S t from the opposite face at t = 1
        return mesh.prism_bar(1.0, 1.0, 3.0, 1.0), P(1.0, 1.0, 2.0, 2.0, 40)
    if name == "limit":      # lambda = -mu: c_P = c_S (the reference's screenUniformLimit problems)
        return mesh.screen_uniform(4), P(1.0, 1.0, -1.0, 1.0, 8)
    if name == "graded":
        return mesh.screen_graded(6, 4), P(1.0, 1.0, 2.0, 1.0, 16)
    raise KeyError(name)


@pytest.mark.parametrize("name,n_gh", [("screen32", 3), ("screen32", 19), ("screen128", 7), ("sphere80", 12),
                                       ("prism", 7), ("limit", 7), ("graded", 7)])
def test_sa_matches_oracle(ebem, oracle, name, n_gh):
    m, prm = _case(name)
    dm = ebem.DeviceMesh(m)
    L = ebem.num_blocks(dm, prm)
    assert L == oracle.num_blocks(m, prm)
    Eg, cnt = ebem.assemble_sa(dm, prm, n_gh, 0, L, count=True)
    Eg = Eg.cpu().numpy()
    assert np.isfinite(Eg).all()
    Eo, cnt_o = oracle.assemble_sa(m, prm, n_gh, 0, L)
    assert cnt == cnt_o
    assert rel(Eg, Eo) <= TOL_F64, f"device vs FP64 restatement {rel(Eg, Eo):.3e}"


GOLDEN = ["screen32_gh3", "screen32_gh7", "screen32_gh12", "screen32_gh19", "screen128_gh7", "sphere80_gh7",
          "sphere80_gh12", "prism28_gh7", "graded48_gh7", "limit32_gh7"]


@pytest.mark.parametrize("case", GOLDEN)
def test_sa_matches_exact_golden(ebem, case):
    """Device blocks against the golden fixtures (tests/golden/make_golden.py):
    the binary128 value of the reference's formulas on a seeded sample of
    400 blocks per case; bar 1e-10 relative."""
    import os
    from conftest import ROOT
    sys_path_golden = os.path.join(ROOT, "tests", "golden")
    import sys
    sys.path.insert(0, sys_path_golden)
    import make_golden
    z = np.load(os.path.join(sys_path_golden, "sa_blocks.npz"))
    name, m, prm, n_gh = [c for c in make_golden.cases() if c[0] == case][0]
    src, fld, lag, exact = z[f"{case}/src"], z[f"{case}/fld"], z[f"{case}/lag"], z[f"{case}/exact"]
    dm = ebem.DeviceMesh(m)
    L = ebem.num_blocks(dm, prm)
    E = ebem.assemble_sa(dm, prm, n_gh, 0, L).cpu().numpy()
    got = np.stack([E[l, 3 * i:3 * i + 3, 3 * j:3 * j + 3] for i, j, l in zip(src, fld, lag)])
    assert rel(got, exact) <= TOL, f"{case}: {rel(got, exact):.3e}"
    assert np.abs(got - exact).max() <= TOL * np.abs(exact).max()


def test_lag_window_and_accumulate(ebem, oracle):
    import torch
    m, prm = _case("sphere80")
    dm = ebem.DeviceMesh(m)
    L = ebem.num_blocks(dm, prm)
    full = ebem.assemble_sa(dm, prm, 7, 0, L).clone()
    a = ebem.assemble_sa(dm, prm, 7, 0, 5).clone()
    b = ebem.assemble_sa(dm, prm, 7, 5, L - 5).clone()
    assert torch.equal(torch.cat([a, b]), full)
    # accumulate: E += block on a pre-filled buffer
    n3 = 3 * m.numberTriangles
    buf = torch.full((L, n3, n3), 0.25, dtype=torch.float64, device="cuda")
    acc = ebem.assemble_sa(dm, prm, 7, 0, L, out=buf, accumulate=True)
    assert torch.allclose(acc, full + 0.25, rtol=0, atol=1e-15)


def test_host_output_matches_device(ebem):
    import torch
    m, prm = _case("screen32")
    dm = ebem.DeviceMesh(m)
    L = ebem.num_blocks(dm, prm)
    dev, cd = ebem.assemble_sa(dm, prm, 7, 0, L, count=True)
    n3 = 3 * m.numberTriangles
    host = torch.empty((L, n3, n3), dtype=torch.float64).pin_memory()
    # the host path assembles in source-row sub-panels: the count sums them
    h, ch = ebem.assemble_sa(dm, prm, 7, 0, L, out=host, count=True)
    assert torch.equal(h, dev.cpu())
    assert ch == cd


def test_host_output_pipeline(ebem):
    """Host outputs are assembled in source-row sub-panels whose copies
    overlap the next sub-panel: accumulation into pageable memory and a row
    panel that starts inside the mesh equal the device results."""
    import torch
    m, prm = _case("screen32")
    dm = ebem.DeviceMesh(m)
    L = ebem.num_blocks(dm, prm)
    n3 = 3 * m.numberTriangles
    dev = ebem.assemble_sa(dm, prm, 7, 0, L).cpu()
    acc = torch.full((L, n3, n3), 0.25, dtype=torch.float64)            # pageable
    h = ebem.assemble_sa(dm, prm, 7, 0, L, out=acc, accumulate=True)
    assert torch.allclose(h, dev + 0.25, rtol=0, atol=1e-15)
    src0, nsrc = 5, 13
    pd = ebem.assemble_sa_panel(dm, prm, 7, 0, L, src0, nsrc).cpu()
    ph = ebem.assemble_sa_panel(dm, prm, 7, 0, L, src0, nsrc, out=torch.empty((L, n3, 3 * nsrc), dtype=torch.float64))
    assert torch.equal(ph, pd)


def test_sphere1280_sampled_blocks(ebem, oracle):
    """Full headline workload on the device; parity on a seeded sample of
    (source, field, lag) blocks plus size-independent properties."""
    from elastodynamicebem_b200 import problem
    w = problem.sphere_workload(7)
    m, prm = w.mesh, w.params
    dm = ebem.DeviceMesh(m)
    L = ebem.num_blocks(dm, prm)
    assert L == 40
    E, cnt = ebem.assemble_sa(dm, prm, 7, 0, L, count=True)
    assert cnt == oracle.count_nonnull(m, prm, L)
    rng = np.random.default_rng(7)
    N = m.numberTriangles
    q = 1500
    src = rng.integers(0, N, q)
    fld = np.where(rng.random(q) < 0.2, src, rng.integers(0, N, q))   # include diagonal blocks
    lag = rng.integers(0, L, q)
    ref = oracle.assemble_sa_pairs(m, prm, 7, src, fld, lag)
    Ec = E.cpu().numpy()
    got = np.stack([Ec[l, 3 * i:3 * i + 3, 3 * j:3 * j + 3] for i, j, l in zip(src, fld, lag)])
    scale = np.abs(Ec).max()
    assert np.abs(got - ref).max() <= TOL_F64 * scale
    assert rel(got, ref) <= TOL_F64
    assert np.isfinite(Ec).all()


def test_large_device_output_lag_windows(ebem):
    """The full 4.7 GB device output of the sphere of 1280 triangles (L = 40)
    equals, bit for bit, its 4-lag windows assembled separately, their
    non-null counts add up to the full count, and accumulating into a copy of
    the blocks doubles them exactly."""
    import torch
    from elastodynamicebem_b200 import problem
    w = problem.sphere_workload(7)
    dm = ebem.DeviceMesh(w.mesh)
    L = ebem.num_blocks(dm, w.params)
    E, cnt = ebem.assemble_sa(dm, w.params, 7, 0, L, count=True)
    total = 0
    for l0 in range(0, L, 4):
        nl = min(4, L - l0)
        Ew, c = ebem.assemble_sa(dm, w.params, 7, l0, nl, count=True)
        assert torch.equal(Ew, E[l0:l0 + nl])
        total += c
        del Ew
    assert total == cnt
    buf = E.transpose(1, 2).clone()                         # a copy in the library's column-major storage
    acc = ebem.assemble_sa(dm, w.params, 7, 0, L, out=buf, accumulate=True)
    assert torch.equal(acc, 2 * E)
