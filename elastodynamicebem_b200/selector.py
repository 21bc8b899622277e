"""Learned quadrature selector: training data, training and use.

The network and every computation on the device are the library's
(``ebem_selector_*``, ``ebem_sa_pair_blocks``, ``ebem_assemble_sa_selected``);
this module samples the training set and strings the calls together.

* Classes are four outer rules, Gauss-Hammer order x congruent
  sub-triangles of the source triangle (GaussHammerComposite.m):
  ``RULES`` = 3 nodes on 1, 7 on 1, 7 on 4 and 7 on 16 sub-triangles; the
  last is the maximal rule, the fallback and the reference that labels and
  errors are measured against.
* Labels come from the plain method's convergence: the blocks of sampled
  (source, field) pairs at every lag under all four rules; a (pair, lag)
  takes the smallest rule whose block is within ``tol`` x sqrt(D_i D_j) of
  the maximal rule's in every entry, D_t the largest entry of triangle t's
  self-interaction block E_0(t, t).  The scale follows the two triangles'
  sizes, so labels learnt on uniform meshes carry over to graded ones (with
  one scale per mesh, the small elements of a graded screen were labelled
  far too loosely: density error 0.27 on the 1024-triangle graded screen).
* Lags during which a wavefront sweeps the pair's distance window take the
  maximal rule without asking the network (``ebem_selector_sweeps``): the
  kernel integral has the kinks of the front crossing the field triangle
  there, and the network's rare confident mistakes on such lags were
  enough to ruin the density on a graded screen (1.8 % of the lags below
  their label gave a density error of 0.54).
* The training set is (pair, lag) samples of the meshes of the benchmark
  configurations 1-4 (screen of 128 triangles, sphere of 1280, prism of
  2800, batch instances) with their time steps and materials, the lags no
  front sweeps.
"""
from __future__ import annotations

import numpy as np
import torch

from . import core, mesh as _mesh, problem

RULES = ((3, 1), (7, 1), (7, 4), (7, 16))
TOL = 1e-10           # label tolerance relative to sqrt(D_i D_j)
THRESHOLD = 0.9       # below this largest probability: the maximal rule


def training_meshes(seed: int = 4):
    """(name, mesh, params) of the meshes of configurations 1-4."""
    out = [("screen_n128", problem.screen_workload().mesh, problem.screen_workload().params)]
    w = problem.sphere_workload(7, 3)
    out.append(("sphere_n1280", w.mesh, w.params))
    b = problem.bar_workload(0.1)
    out.append(("prism_n2800", b.mesh, b.params))
    inst = problem.batch_workload(count=64, seed=seed)
    rng = np.random.default_rng(seed)
    for k in rng.choice(len(inst), 4, replace=False):
        out.append(tuple(inst[int(k)]))
    return out


def diagonal_scales(dm: core.DeviceMesh, prm, rules=RULES) -> torch.Tensor:
    """D_t = largest entry of E_0(t, t) on the maximal rule, every triangle t."""
    i = torch.arange(dm.N, dtype=torch.int32, device="cuda")
    pairs = torch.stack([i, i], 1).contiguous()
    b = core.sa_pair_blocks(dm, prm, rules[-1][0], rules[-1][1], pairs, 1)      # (N, 1, 6)
    return b.abs().amax(dim=(1, 2))


def samples_for_mesh(m, prm, n_samples: int, rules=RULES, tol: float = TOL, seed: int = 0):
    """(features, labels, samples) of about n_samples seeded (pair, lag)
    samples of one mesh: uniformly drawn pairs, every non-null lag of each."""
    dm = core.DeviceMesh(m)
    L = core.num_blocks(dm, prm)
    rng = np.random.default_rng(seed)
    N = dm.N
    # most non-null lags are swept by a front: draw enough pairs for n_samples free ones
    npairs = max(64, int(12 * n_samples / max(1, 0.5 * L)))
    pairs = np.stack([rng.integers(0, N, npairs), rng.integers(0, N, npairs)], 1)
    tp = torch.tensor(pairs, dtype=torch.int32, device="cuda")
    blocks = torch.stack([core.sa_pair_blocks(dm, prm, n, s, tp, L) for n, s in rules])   # (4, P, L, 6)
    nonnull = blocks[-1].abs().amax(dim=2) > 0                                              # (P, L)
    pidx, lidx = torch.nonzero(nonnull, as_tuple=True)
    cand = torch.stack([tp[pidx, 0], tp[pidx, 1], lidx.to(torch.int32)], 1).contiguous()
    # the network decides only lags that no wavefront sweeps (the others take
    # the maximal rule at inference): train on those
    free = core.selector_sweeps(dm, prm, cand) == 0
    pidx, lidx, cand = pidx[free], lidx[free], cand[free]
    keep = torch.randperm(pidx.numel(), generator=torch.Generator().manual_seed(seed))[:n_samples].cuda()
    pidx, lidx = pidx[keep], lidx[keep]
    smp = cand[keep].contiguous()
    b = blocks[:, pidx, lidx, :].contiguous()                                               # (4, n, 6)
    D = diagonal_scales(dm, prm, rules)
    scales = torch.sqrt(D[smp[:, 0].long()] * D[smp[:, 1].long()])
    y = core.selector_labels(b, tol, 1.0, scales)
    x = core.selector_features(dm, prm, smp)
    dm.close()
    return x, y, smp


def training_set(n_total: int = 200_000, rules=RULES, tol: float = TOL, seed: int = 4):
    """200k seeded (pair, lag) samples of the configuration 1-4 meshes,
    shares equal per configuration (configuration 4's split over its
    instances); returns (features, labels) on the device, shuffled."""
    meshes = training_meshes(seed)
    share = {0: n_total // 4, 1: n_total // 4, 2: n_total // 4}
    rest = n_total - 3 * (n_total // 4)
    X, Y = [], []
    for k, (name, m, prm) in enumerate(meshes):
        n = share.get(k, rest // (len(meshes) - 3))
        x, y, _ = samples_for_mesh(m, prm, n, rules, tol, seed + k)
        X.append(x)
        Y.append(y)
    X, Y = torch.cat(X), torch.cat(Y)
    perm = torch.randperm(X.shape[0], generator=torch.Generator().manual_seed(seed)).cuda()
    return X[perm].contiguous(), Y[perm].contiguous()


def train(X, Y, epochs: int = 30, batch: int = 512, lr: float = 3e-3, seed: int = 7):
    """Parameters trained on the device; returns (params, per-epoch loss)."""
    params = core.selector_init(seed=seed)
    losses = core.selector_train(params, X, Y, epochs=epochs, batch=batch, lr=lr, seed=seed + 2)
    return params, losses


def assemble(params, dm: core.DeviceMesh, prm, rules=RULES, threshold: float = THRESHOLD, lag0: int = 0,
             nlag: int | None = None, out=None, prec: int = core.PREC_FP64):
    """Inference over every (pair, lag) and the assembly of each on its
    class's rule; returns (E, non-null lags per class)."""
    cls, _ = core.selector_infer(params, dm, prm, threshold, lag0, nlag)
    return core.assemble_sa_selected(dm, prm, cls, rules, lag0, nlag, out=out, prec=prec)
