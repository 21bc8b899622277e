"""Learned quadrature selector on the device: features and the network's
gradient against the CPU restatement (oracle/selector_oracle.py), the
convergence labels against the plain assemblies they come from, and a
training run whose gain over the plain method is measured: time and
time-marched density error of the selector-driven assembly against the plain
assembly on the maximal (19-node) rule and on the 7-node rule."""
import os
import sys

import numpy as np
import pytest

from conftest import cuda_available

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import selector_oracle as SO  # noqa: E402

pytestmark = pytest.mark.gpu

TAU = 1e-3            # label tolerance, relative to max |E| of the maximal rule


@pytest.fixture(scope="module")
def ebem():
    if not cuda_available():
        pytest.skip("no CUDA device")
    import elastodynamicebem_b200.core as core
    return core


def test_features_match_oracle(ebem):
    from elastodynamicebem_b200 import mesh, problem
    m, prm = mesh.icosphere(1), problem.ProblemParams(1.0, 1.0, 1.0, 1.0, 40)
    dm = ebem.DeviceMesh(m)
    f = ebem.selector_features(dm, prm).cpu().numpy()
    assert np.abs(f - SO.features(m, prm)).max() <= 1e-5


def test_gradient_matches_oracle(ebem):
    import torch
    rng = np.random.default_rng(1)
    n = 1000
    x = rng.normal(size=(n, 12)).astype(np.float32)
    y = rng.integers(0, 4, n).astype(np.int32)
    params = ebem.selector_init(seed=3)
    g, loss = ebem.selector_grad(params, torch.tensor(x, device="cuda"), torch.tensor(y, device="cuda"))
    lo, go = SO.loss_and_grad(params.cpu().numpy().astype(np.float64), x.astype(np.float64), y)
    g = g.cpu().numpy()
    assert abs(loss - lo) <= 1e-5 * abs(lo)
    assert np.linalg.norm(g - go) <= 1e-4 * np.linalg.norm(go)


def test_labels_match_plain_assemblies(ebem):
    import torch
    from elastodynamicebem_b200 import mesh, problem
    m, prm = mesh.screen_uniform(4), problem.ProblemParams(1.0, 1.0, 2.0, 1.0, 20)
    dm = ebem.DeviceMesh(m)
    N = m.numberTriangles
    lab = ebem.selector_labels(dm, prm, TAU).cpu().numpy()
    L = ebem.num_blocks(dm, prm)
    E = {r: ebem.assemble_sa(dm, prm, r, 0, L).clone().view(L, N, 3, N, 3) for r in (3, 7, 12, 19)}
    scale = float(E[19].abs().max())
    err = {r: (E[r] - E[19]).abs().amax(dim=(0, 2, 4)).cpu().numpy() for r in (3, 7, 12)}   # [i, j]
    ref = np.full((N, N), 3)
    for q, r in reversed(list(enumerate((3, 7, 12)))):
        ref[err[r] <= TAU * scale] = q
    assert np.array_equal(lab, ref.T.reshape(-1))       # pair p = j * N + i


def test_selected_assembly_per_class(ebem):
    """Each pair is assembled on the rule of its class: one class everywhere
    equals the plain assembly on that rule, and a mixed class map equals the
    plain blocks of each pair's rule."""
    import torch
    from elastodynamicebem_b200 import mesh, problem
    m, prm = mesh.icosphere(1), problem.ProblemParams(1.0, 1.0, 1.0, 1.0, 40)
    dm = ebem.DeviceMesh(m)
    N, L = m.numberTriangles, ebem.num_blocks(ebem.DeviceMesh(m), prm)
    plain = {r: ebem.assemble_sa(dm, prm, r, 0, L).clone().view(L, N, 3, N, 3) for r in (3, 7, 12, 19)}
    for q, r in enumerate((3, 7, 12, 19)):
        cls = torch.full((N * N,), q, dtype=torch.int32, device="cuda")
        E, counts = ebem.assemble_sa_selected(dm, prm, cls, 0, L)
        assert counts[q] == N * N
        assert float((E.clone().view(L, N, 3, N, 3) - plain[r]).norm() / plain[r].norm()) <= 1e-12
    cls = torch.tensor(np.random.default_rng(2).integers(0, 4, N * N), dtype=torch.int32, device="cuda")
    E, counts = ebem.assemble_sa_selected(dm, prm, cls, 0, L)
    E = E.clone().view(L, N, 3, N, 3)
    pick = cls.view(N, N).T.long()                        # [i, j] (pair p = j * N + i)
    ref = torch.zeros_like(E)
    for q, r in enumerate((3, 7, 12, 19)):
        mask = (pick == q)[None, :, None, :, None]
        ref = torch.where(mask, plain[r], ref)
    assert float((E - ref).norm() / ref.norm()) <= 1e-12
    assert sum(counts) == N * N


def _timed(fn, reps=3):
    import torch
    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        out = fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps, out


def test_trained_selector_gain(ebem):
    """Train on pairs of screens and coarse spheres; use the network on a finer
    sphere (not seen in training) and measure what it gains over the plain
    method: assembly time and time-marched density error against the plain
    assembly on the maximal rule (19 nodes) and on the 7-node rule."""
    import torch
    from elastodynamicebem_b200 import mesh, problem
    train = [(mesh.screen_uniform(8), problem.ProblemParams(1.0, 1.0, 2.0, 1.0, 20)),
             (mesh.screen_graded(6, 4), problem.ProblemParams(1.0, 1.0, 2.0, 1.0, 16)),
             (mesh.icosphere(1), problem.ProblemParams(1.0, 1.0, 1.0, 1.0, 40)),
             (mesh.icosphere(2), problem.ProblemParams(1.0, 1.0, 1.0, 1.0, 40))]
    X, Y = [], []
    for m, prm in train:
        dm = ebem.DeviceMesh(m)
        X.append(ebem.selector_features(dm, prm))
        Y.append(ebem.selector_labels(dm, prm, TAU))
    X, Y = torch.cat(X), torch.cat(Y)
    perm = torch.randperm(X.shape[0], generator=torch.Generator().manual_seed(5)).cuda()
    X, Y = X[perm].contiguous(), Y[perm].contiguous()
    ntr = int(0.85 * X.shape[0])
    params = ebem.selector_init(seed=7)
    _, loss0 = ebem.selector_grad(params, X[:ntr], Y[:ntr])
    losses = ebem.selector_train(params, X[:ntr], Y[:ntr], epochs=25, batch=512, lr=3e-3, seed=9)
    assert losses[-1] < 0.5 * loss0 and losses[-1] <= losses[0]
    # held-out accuracy against the majority class
    _, lo_test = ebem.selector_grad(params, X[ntr:], Y[ntr:])
    counts = torch.bincount(Y[ntr:].long(), minlength=4).float()
    prior = counts / counts.sum()
    base_loss = float(-(prior * torch.log(torch.clamp(prior, min=1e-12))).sum())
    assert lo_test < base_loss
    # gain on an unseen mesh: sphere of 1280 triangles, GH7 time and error for scale
    w = problem.sphere_workload(7, 3)
    dm = ebem.DeviceMesh(w.mesh)
    L = ebem.num_blocks(dm, w.params)
    classes = ebem.selector_infer(params, dm, w.params, 0.9)
    buf = torch.empty((L, 3 * dm.N, 3 * dm.N), dtype=torch.float64, device="cuda")
    t_sel, (E_sel, per_class) = _timed(lambda: ebem.assemble_sa_selected(dm, w.params, classes, 0, L, out=buf))
    E_sel = E_sel.clone()
    t19, E19 = _timed(lambda: ebem.assemble_sa(dm, w.params, 19, 0, L, out=buf))
    E19 = E19.clone()
    t7, E7 = _timed(lambda: ebem.assemble_sa(dm, w.params, 7, 0, L, out=buf))
    E7 = E7.clone()
    b = ebem.rhs(dm, w.params, 19, w.datum)
    phi19 = ebem.march(E19, b)
    phi_sel = ebem.march(E_sel, b)
    phi7 = ebem.march(E7, ebem.rhs(dm, w.params, 7, w.datum))
    err_sel = float((phi_sel - phi19).norm() / phi19.norm())
    err7 = float((phi7 - phi19).norm() / phi19.norm())
    print(f"\nselector on sphere N=1280: classes {per_class}; assembly {t_sel:.1f} ms vs GH19 {t19:.1f} ms "
          f"({t19 / t_sel:.2f}x) and GH7 {t7:.1f} ms; density error vs GH19: selector {err_sel:.2e}, GH7 {err7:.2e}")
    # What the network gains is measured and printed, not assumed: with the
    # outer rules' slow convergence at the wavefronts it need not beat the
    # plain rules (the measured trade-off is recorded with the design notes).
    assert sum(per_class) == dm.N ** 2
    assert np.isfinite(err_sel) and t_sel > 0
