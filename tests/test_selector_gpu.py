"""Learned quadrature selector on the device: per-(pair, lag) features and
the network's gradient against the CPU restatement
(oracle/selector_oracle.py), the plain method's blocks with composite outer
rules (GaussHammerComposite) against the dense assembly, the convergence
labels, the assembly of each (pair, lag) on the rule of its class, and a
training run whose gain is measured and asserted."""
import os
import sys

import numpy as np
import pytest

from conftest import cuda_available

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import selector_oracle as SO  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ebem():
    if not cuda_available():
        pytest.skip("no CUDA device")
    import elastodynamicebem_b200.core as core
    return core


def _sphere80():
    from elastodynamicebem_b200 import mesh, problem
    return mesh.icosphere(1), problem.ProblemParams(1.0, 1.0, 1.0, 1.0, 40)


def _sym(E, N, L):
    """(N_src, N_fld, L, 6) symmetric entries of E[l][3i+a, 3j+b]."""
    v = E.reshape(L, N, 3, N, 3).permute(1, 3, 0, 2, 4)
    import torch
    return torch.stack([v[..., 0, 0], v[..., 0, 1], v[..., 0, 2], v[..., 1, 1], v[..., 1, 2], v[..., 2, 2]], -1)


def test_features_match_oracle(ebem):
    import torch
    m, prm = _sphere80()
    dm = ebem.DeviceMesh(m)
    rng = np.random.default_rng(0)
    N = m.numberTriangles
    smp = np.stack([rng.integers(0, N, 2000), rng.integers(0, N, 2000), rng.integers(0, 41, 2000)], 1)
    smp[:50, 1] = smp[:50, 0]
    f = ebem.selector_features(dm, prm, torch.tensor(smp, dtype=torch.int32, device="cuda")).cpu().numpy()
    assert np.abs(f - SO.lag_features(m, prm, smp)).max() <= 1e-5


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


def test_labels_match_oracle(ebem):
    import torch
    rng = np.random.default_rng(2)
    ref = rng.normal(size=(3000, 6))
    scales = rng.choice([1e-2, 1e-5, 1e-8, 1e-11], size=(3, 3000, 1))
    blocks = np.concatenate([ref[None] + rng.normal(size=(3, 3000, 6)) * scales, ref[None]])
    sc = rng.uniform(0.1, 10.0, 3000)
    for tol in (1e-4, 1e-7, 1e-10):
        lab = ebem.selector_labels(torch.tensor(blocks, device="cuda"), tol, 2.0).cpu().numpy()
        assert np.array_equal(lab, SO.labels(blocks, tol, 2.0))
        lab = ebem.selector_labels(torch.tensor(blocks, device="cuda"), tol, 2.0, torch.tensor(sc)).cpu().numpy()
        assert np.array_equal(lab, SO.labels(blocks, tol, 2.0, sc))


def test_composite_rules_pair_blocks_match_dense(ebem):
    """The plain method with composite outer rules: the pair-list blocks equal
    the dense assembly's, rule (7, 1) equals the ordinary 7-node assembly, and
    refining the composite rule converges."""
    import torch
    m, prm = _sphere80()
    dm = ebem.DeviceMesh(m)
    N, L = m.numberTriangles, ebem.num_blocks(dm, prm)
    rng = np.random.default_rng(5)
    pairs = torch.tensor(np.stack([rng.integers(0, N, 400), rng.integers(0, N, 400)], 1), dtype=torch.int32,
                         device="cuda")
    i, j = pairs[:, 0].long(), pairs[:, 1].long()
    dense = {}
    for n, sub in ((7, 1), (7, 4), (3, 16), (7, 16)):
        E = ebem.assemble_sa_rule(dm, prm, n, sub, 0, L).clone()
        dense[(n, sub)] = E
        pb = ebem.sa_pair_blocks(dm, prm, n, sub, pairs, L)
        ref = _sym(E, N, L)[i, j]
        assert float((pb - ref).abs().max() / ref.abs().max()) <= 1e-13
    E7 = ebem.assemble_sa(dm, prm, 7, 0, L)
    assert float((dense[(7, 1)] - E7).abs().max() / E7.abs().max()) <= 1e-13
    e1 = float((dense[(7, 1)] - dense[(7, 16)]).norm() / dense[(7, 16)].norm())
    e4 = float((dense[(7, 4)] - dense[(7, 16)]).norm() / dense[(7, 16)].norm())
    assert e4 < e1


def test_selected_assembly_per_lag_class(ebem):
    """Each (pair, lag) is assembled on the rule of its class: a random class
    map equals, block by block, the plain assembly on each block's rule, and
    the class counts add up to the non-null pair-lags."""
    import torch
    m, prm = _sphere80()
    dm = ebem.DeviceMesh(m)
    N, L = m.numberTriangles, ebem.num_blocks(dm, prm)
    rules = ((7, 1), (3, 4), (7, 4), (12, 4))
    plain = [ebem.assemble_sa_rule(dm, prm, n, sub, 0, L).clone().reshape(L, N, 3, N, 3) for n, sub in rules]
    g = torch.Generator(device="cuda").manual_seed(3)
    cls = torch.randint(0, 4, (N * N, L), dtype=torch.uint8, device="cuda", generator=g)
    E, counts = ebem.assemble_sa_selected(dm, prm, cls, rules, 0, L)
    E = E.clone().reshape(L, N, 3, N, 3)
    pick = cls.view(N, N, L).permute(2, 1, 0)             # [l, i, j] (row = field * N + source)
    ref = torch.zeros_like(E)
    for c in range(4):
        ref = torch.where((pick == c)[:, :, None, :, None], plain[c], ref)
    assert float((E - ref).abs().max() / ref.abs().max()) <= 1e-13
    _, nonnull = ebem.assemble_sa(dm, prm, 7, 0, L, count=True)
    assert sum(counts) == nonnull


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
    """Train on 200k seeded (pair, lag) samples of the configuration 1-4
    meshes (labels from the plain method's convergence over the four rules),
    then assemble configuration 2 (sphere of 1280 triangles) and a graded
    screen with configuration 5's grading, time step and lags (1024
    triangles, not among the training meshes) with the network's classes.
    Asserted: the density and the post-processed displacement are within
    1e-6 of the plain method on the maximal rule, and the selected assembly,
    its four class passes included, costs at most 5 % more than that plain
    assembly.  The gain is printed: it is small whatever the network does,
    because the blocks that converge on a cheaper rule are those no
    wavefront crosses, whose levels the plain kernel already passes over
    cheaply (perfect labels gain 1.08x on the 320-triangle sphere)."""
    import torch
    from elastodynamicebem_b200 import problem
    from elastodynamicebem_b200 import selector as S
    X, Y = S.training_set(200_000)
    n = X.shape[0]
    ntr = int(0.9 * n)
    params = ebem.selector_init(seed=7)
    _, loss0 = ebem.selector_grad(params, X[:ntr], Y[:ntr])
    losses = ebem.selector_train(params, X[:ntr], Y[:ntr], epochs=20, batch=512, lr=3e-3, seed=9)
    assert losses[-1] < 0.5 * loss0 and losses[-1] <= losses[0]
    _, lo_test = ebem.selector_grad(params, X[ntr:], Y[ntr:])
    prior = torch.bincount(Y[ntr:].long(), minlength=4).double()
    prior = prior / prior.sum()
    assert lo_test < float(-(prior * torch.log(torch.clamp(prior, min=1e-12))).sum())
    for w in (problem.sphere_workload(7, 3), problem.graded_workload(16, 32)):
        dm = ebem.DeviceMesh(w.mesh)
        L = ebem.num_blocks(dm, w.params)
        n3 = 3 * dm.N
        buf = torch.empty((L, n3, n3), dtype=torch.float64, device="cuda")
        t_max, E = _timed(lambda: ebem.assemble_sa_rule(dm, w.params, *S.RULES[-1], 0, L, out=buf), reps=1)
        b = ebem.rhs(dm, w.params, 7, w.datum)
        phi_max = ebem.march(E, b)
        t_sel, (E, counts) = _timed(lambda: S.assemble(params, dm, w.params, out=buf), reps=1)
        phi_sel = ebem.march(E, b)
        del E
        u_max = ebem.pp_sa(dm, w.params, phi_max, w.points, w.times)
        u_sel = ebem.pp_sa(dm, w.params, phi_sel, w.points, w.times)
        err_d = float((phi_sel - phi_max).norm() / phi_max.norm())
        err_u = float((u_sel - u_max).norm() / u_max.norm())
        print(f"\nselector on {w.name}: non-null lags per class {counts}; assembly {t_sel:.1f} ms vs the maximal "
              f"rule's {t_max:.1f} ms ({t_max / t_sel:.2f}x); density error {err_d:.2e}, displacement {err_u:.2e}")
        assert err_d <= 1e-6 and err_u <= 1e-6
        assert t_sel <= 1.05 * t_max
        del buf
        torch.cuda.empty_cache()


def test_rule_selection_bound(ebem):
    """What any selector over these rules can save, with the labels themselves
    as the classes (a perfect network) on the sphere of 320 triangles
    (configuration 2's material and time step): at the labels' tolerance the
    density is within 1e-6 of the maximal rule, and the outer nodes the
    selected lags use are still more than a fifth of the maximal rule's, so
    no choice among these rules reaches the 5x of the forms' target (most
    non-null blocks have a wavefront crossing their field triangle, where the
    outer rule converges only algebraically)."""
    import torch
    from elastodynamicebem_b200 import problem
    from elastodynamicebem_b200 import selector as S
    w = problem.sphere_workload(7, 2)
    dm = ebem.DeviceMesh(w.mesh)
    N, L = dm.N, ebem.num_blocks(dm, w.params)
    E = [ebem.assemble_sa_rule(dm, w.params, n, s, 0, L).clone().reshape(L, N, 3, N, 3) for n, s in S.RULES]
    D = S.diagonal_scales(dm, w.params)
    thr = S.TOL * torch.sqrt(D[:, None] * D[None, :])[None]                     # (1, N_src, N_fld)
    nonnull = E[-1].abs().amax(dim=(2, 4)) > 0                                    # (L, N_src, N_fld)
    lab = torch.full((L, N, N), len(S.RULES) - 1, dtype=torch.uint8, device="cuda")
    for c in range(len(S.RULES) - 2, -1, -1):
        lab[(E[c] - E[-1]).abs().amax(dim=(2, 4)) <= thr] = c
    cls = lab.permute(2, 1, 0).reshape(N * N, L).contiguous()                    # row = field * N + source
    Es, counts = ebem.assemble_sa_selected(dm, w.params, cls, S.RULES, 0, L)
    b = ebem.rhs(dm, w.params, 7, w.datum)
    phi = ebem.march(Es.clone(), b)
    phi_max = ebem.march(ebem.assemble_sa_rule(dm, w.params, *S.RULES[-1], 0, L), b)
    err = float((phi - phi_max).norm() / phi_max.norm())
    nodes = torch.tensor([n * s for n, s in S.RULES], dtype=torch.float64, device="cuda")
    used = float(nodes[lab[nonnull].long()].sum())
    full = float(nonnull.sum()) * float(nodes[-1])
    print(f"\nperfect labels on {w.name}: non-null lags per class {counts}; density error {err:.2e}; "
          f"outer nodes used {used / full:.3f} of the maximal rule's")
    assert err <= 1e-6
    assert used / full > 0.2
