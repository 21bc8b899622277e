"""Each hot-path row on the device beside the reference's own implementation
of it on the same inputs: the reference's CUDA kernels (kernelGHC / kernelV,
kernelK, kernelG and kernelP, compiled from the reference's sources into
oracle/_ref and run on this GPU) or, for the rows whose reference code is
MATLAB on the CPU, the oracle's C++ restatement on all host cores.  Every row
asserts parity with that implementation and records both times; the last
test prints the table (run with ``pytest -s``).

Timing: the device paths with CUDA events over 3 calls after one warm-up
(device-resident inputs and outputs); the reference kernels with CUDA events
around their launch (their host copies excluded); the CPU restatement with
the wall clock."""
import os
import sys
import time

import numpy as np
import pytest

from conftest import cuda_available

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import oracle as O  # noqa: E402

pytestmark = pytest.mark.gpu

ROWS = []


@pytest.fixture(scope="module")
def ebem():
    if not cuda_available():
        pytest.skip("no CUDA device")
    import elastodynamicebem_b200.core as core
    return core


def dev_ms(fn, reps=3):
    import torch
    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def cpu_ms(fn):
    t0 = time.perf_counter()
    out = fn()
    return 1e3 * (time.perf_counter() - t0), out


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def record(row, case, ours, ref, kind, err):
    ROWS.append((row, case, ours, ref, kind, err))


@pytest.fixture(scope="module")
def sphere(ebem):
    from elastodynamicebem_b200 import problem
    w = problem.sphere_workload(7, 2)
    dm = ebem.DeviceMesh(w.mesh)
    return w, dm, ebem.num_blocks(dm, w.params)


@pytest.fixture(scope="module")
def bar(ebem):
    from elastodynamicebem_b200 import mesh, problem
    m, prm = mesh.prism_bar(1.0, 1.0, 3.0, 0.25), problem.ProblemParams(1.0, 1.0, 2.0, 2.0, 40)
    dm = ebem.DeviceMesh(m)
    return m, prm, dm, ebem.num_blocks_dir(dm, prm)


def test_row_sa_assembly(ebem, sphere):
    import torch
    w, dm, L = sphere
    n3 = 3 * dm.N
    buf = torch.empty((L, n3, n3), dtype=torch.float64, device="cuda")
    ours = dev_ms(lambda: ebem.assemble_sa(dm, w.params, w.n_gh, 0, L, out=buf))
    E = ebem.assemble_sa(dm, w.params, w.n_gh, 0, L, out=buf).cpu().numpy()
    ref, (Eo, _) = cpu_ms(lambda: O.assemble_sa(w.mesh, w.params, w.n_gh, 0, L))
    err = rel(E, Eo)
    record("a4-a12 SA assembly", f"sphere N={dm.N}, L={L}, GH7", ours, ref, f"C++ restatement, {os.cpu_count()} cores", err)
    assert err <= 1e-7          # the restatement's own FP64 noise (edge form vs law-of-cosines form)


def test_row_ghc(ebem, sphere):
    w, dm, L = sphere
    if not O.ref_ghc_available():
        pytest.skip("reference kernels not built")
    ours = dev_ms(lambda: ebem.assemble_ghc(dm, w.params, 7, 16, 3, 0, L, sa_diagonal=False))
    E = ebem.assemble_ghc(dm, w.params, 7, 16, 3, 0, L, sa_diagonal=False).cpu().numpy()
    Er = O.ref_ghc(w.mesh, w.params, 7, 16, 3, L)
    err = rel(E, Er)
    record("a14 numerical inner (kernelGHC)", f"sphere N={dm.N}, L={L}, rule 7/16/3", ours, O.ref_kernel_ms("ghc"),
           "reference kernelGHC on this GPU", err)
    assert err <= 1e-10


def test_row_rhs(ebem, sphere):
    w, dm, L = sphere
    ours = dev_ms(lambda: ebem.rhs(dm, w.params, w.n_gh, w.datum))
    b = ebem.rhs(dm, w.params, w.n_gh, w.datum).cpu().numpy()
    ref, bo = cpu_ms(lambda: O.rhs(w.mesh, w.params, w.n_gh, w.datum))
    err = rel(b.T, bo)
    record("a15 right-hand side", f"sphere N={dm.N}, nT={w.params.nT}", ours, ref, "C++ restatement, 1 core", err)
    assert err <= 1e-13


def test_row_march(ebem, sphere):
    w, dm, L = sphere
    E = ebem.assemble_sa(dm, w.params, w.n_gh, 0, L).clone()
    b = ebem.rhs(dm, w.params, w.n_gh, w.datum)
    ours = dev_ms(lambda: ebem.march(E, b))
    phi = ebem.march(E, b).cpu().numpy()
    ref, phio = cpu_ms(lambda: O.march(E.cpu().numpy(), b.cpu().numpy().T))
    err = rel(phi.T, phio)
    record("a16 time marching", f"sphere N={dm.N}, L={L}, nT={w.params.nT}", ours, ref, "C++ restatement (LU), 1 core", err)
    assert err <= 1e-10


def test_row_pp_sa(ebem, sphere):
    w, dm, L = sphere
    phi, _ = ebem.timemarch_sa(dm, w.params, w.n_gh, w.datum)
    pts, tms = w.points[:64], w.times
    ours = dev_ms(lambda: ebem.pp_sa(dm, w.params, phi, pts, tms))
    u = ebem.pp_sa(dm, w.params, phi, pts, tms).cpu().numpy()
    ref, uo = cpu_ms(lambda: O.pp_sa(w.mesh, w.params, phi.cpu().numpy().T, pts, tms))
    err = rel(u, np.asarray(uo).transpose(2, 1, 0))          # oracle: (3, points, times)
    record("a17 post-processing (closed form)", f"sphere N={dm.N}, {len(pts)} points x {len(tms)} times", ours, ref,
           f"C++ restatement, {os.cpu_count()} cores", err)
    assert err <= 1e-10


def test_row_pp_numerical(ebem, sphere):
    """a17's numerical half: kernelLayer (many points at one time, the density
    contraction in the kernel) and kernelSP (one point, its times) against
    the reference's kernels on this GPU, rule 16 x 3 (main.m:135-141 "GPU 16 3")."""
    w, dm, L = sphere
    if not O.ref_pp_available():
        pytest.skip("reference kernels not built")
    phi, _ = ebem.timemarch_sa(dm, w.params, w.n_gh, w.datum)
    ph = phi.cpu().numpy().T
    pts = w.points[:64]
    t = w.times[-1]
    ours = dev_ms(lambda: ebem.pp_gpu(dm, w.params, phi, pts, [t], 16, 3, 1))
    ul = ebem.pp_gpu(dm, w.params, phi, pts, [t], 16, 3, 1).cpu().numpy()[0].T
    ulr, ref = O.ref_pp_layer(w.mesh, w.params, ph, pts, t, 16, 3)
    err = rel(ul, ulr)
    record("a17 numerical post-processing (kernelLayer)", f"sphere N={dm.N}, {len(pts)} points at t={t:g}", ours, ref,
           "reference kernelLayer on this GPU", err)
    assert err <= 1e-12
    x, tms = w.points[5], w.times
    ours = dev_ms(lambda: ebem.pp_gpu(dm, w.params, phi, x[None], tms, 16, 3, 0))
    us = ebem.pp_gpu(dm, w.params, phi, x[None], tms, 16, 3, 0).cpu().numpy()[:, 0]
    ref, urs = 0.0, []
    for tt in tms:
        uu, ms = O.ref_pp_sp(w.mesh, w.params, ph, x, tt, 16, 3)
        urs.append(uu)
        ref += ms
    err = rel(us, np.stack(urs))
    record("a17 numerical post-processing (kernelSP)", f"sphere N={dm.N}, 1 point x {len(tms)} times", ours, ref,
           "reference kernelSP on this GPU, one launch per (x, t), host sums excluded", err)
    assert err <= 1e-12


def test_row_kernel_k(ebem, bar):
    m, prm, dm, (LV, LK) = bar
    if not O.ref_dir_available():
        pytest.skip("reference kernels not built")
    ours = dev_ms(lambda: ebem.assemble_k(dm, prm, 7, 4, 3, 0, 0, LK))
    K = ebem.assemble_k(dm, prm, 7, 4, 3, 0, 0, LK).cpu().numpy()
    Kr = O.ref_k(m, prm, 7, 4, 3, LK)
    err = rel(K, Kr)
    record("a18 double layer (kernelK)", f"bar N={m.numberTriangles}, Nv={m.number_nodes}, L_K={LK}, rule 7/4/3",
           ours, O.ref_kernel_ms("k"), "reference kernelK on this GPU", err)
    assert err <= 1e-10


def test_row_kernel_v(ebem, bar):
    m, prm, dm, (LV, LK) = bar
    if not O.ref_ghc_available():
        pytest.skip("reference kernels not built")
    ours = dev_ms(lambda: ebem.assemble_ghc(dm, prm, 7, 4, 3, 0, LV, sa_diagonal=False))
    V = ebem.assemble_ghc(dm, prm, 7, 4, 3, 0, LV, sa_diagonal=False).cpu().numpy()
    Vr = O.ref_ghc(m, prm, 7, 4, 3, LV)
    err = rel(V, Vr)
    record("a18 single layer off the diagonal (kernelV = kernelGHC)",
           f"bar N={m.numberTriangles}, L_V={LV}, rule 7/4/3", ours, O.ref_kernel_ms("ghc"),
           "reference kernelV on this GPU", err)
    assert err <= 1e-10


def test_row_pp_dir(ebem, bar):
    import torch
    from elastodynamicebem_b200 import problem
    m, prm, dm, (LV, LK) = bar
    if not O.ref_dir_available():
        pytest.skip("reference kernels not built")
    rng = np.random.default_rng(3)
    pts = np.column_stack([rng.uniform(0.1, 0.9, 16), rng.uniform(0.1, 0.9, 16), rng.uniform(0.2, 2.8, 16)])
    tms = np.array([0.5, 1.0, 1.5, 2.0])
    gV = torch.tensor(problem.bar_neumann(m, prm, 3.0), device="cuda")
    u = torch.zeros((prm.nT, 3 * m.number_nodes), dtype=torch.float64, device="cuda")
    ours = dev_ms(lambda: ebem.pp_dir(dm, prm, 4, 3, gV, u, pts, tms))
    ref = 0.0
    for t in tms:
        for x in pts:
            O.ref_pp_dir(m, prm, 4, 3, x, t)
            ref += O.ref_kernel_ms("g") + O.ref_kernel_ms("p")
    x, t = pts[0], tms[-1]
    G, P = ebem.pp_dir_matrices(dm, prm, 4, 3, x, t)
    Gr, Pr = O.ref_pp_dir(m, prm, 4, 3, x, t)
    err = max(rel(G, Gr), rel(P, Pr))
    record("a19 direct post-processing (kernelG + kernelP)",
           f"bar N={m.numberTriangles}, {len(pts)} points x {len(tms)} times", ours, ref,
           "reference kernelG + kernelP on this GPU, one launch pair per (x, t)", err)
    assert err <= 1e-12


def test_row_dn_marching(ebem, bar):
    import torch
    from elastodynamicebem_b200 import problem
    from test_direct_gpu import _march_dn_numpy
    m, prm, dm, (LV, LK) = bar
    V = ebem.assemble_v(dm, prm, 7, 4, 3, 16, 0, LV).clone()
    K = ebem.assemble_k(dm, prm, 7, 4, 3, 16, 0, LK).clone()
    gV = torch.tensor(problem.bar_neumann(m, prm, 3.0), device="cuda")
    ours = dev_ms(lambda: ebem.march_dn(dm, prm, V, K, gV))
    u = ebem.march_dn(dm, prm, V, K, gV).cpu().numpy()
    ref, uo = cpu_ms(lambda: _march_dn_numpy(m, prm, V.cpu().numpy(), K.cpu().numpy(), gV.cpu().numpy()))
    err = rel(u, uo)
    record("a18 DN marching", f"bar N={m.numberTriangles}, Nv={m.number_nodes}, nT={prm.nT}", ours, ref,
           "the reference's per-step least squares in numpy/LAPACK (BEMenerg_dir_timeMarchingN.m:268-299)", err)
    assert err <= 1e-9


def test_zz_print_table():
    if not ROWS:
        pytest.skip("no rows measured")
    print("\n| row | case | ours (ms) | reference (ms) | reference path | speed-up | rel. difference |")
    print("|---|---|---|---|---|---|---|")
    for row, case, ours, ref, kind, err in ROWS:
        print(f"| {row} | {case} | {ours:.2f} | {ref:.2f} | {kind} | {ref / ours:.1f}x | {err:.1e} |")
