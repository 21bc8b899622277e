"""The selector's CPU restatement (oracle/selector_oracle.py), pinned by
finite differences: its analytic gradient is what the device gradient kernel
is checked against."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import selector_oracle as S  # noqa: E402


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = rng.normal(scale=0.3, size=S.NPARAMS)
    x = rng.normal(size=(40, S.F))
    y = rng.integers(0, S.C, 40)
    loss, g = S.loss_and_grad(p, x, y)
    for k in rng.choice(S.NPARAMS, 60, replace=False):
        e = np.zeros(S.NPARAMS); e[k] = 1e-6
        fd = (S.loss_and_grad(p + e, x, y)[0] - S.loss_and_grad(p - e, x, y)[0]) / 2e-6
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(g[k]))
    assert S.NPARAMS == 5252


def test_features_finite_and_bounded():
    from elastodynamicebem_b200 import mesh, problem
    m = mesh.icosphere(1)
    rng = np.random.default_rng(3)
    n = m.numberTriangles
    samples = np.stack([rng.integers(0, n, 500), rng.integers(0, n, 500), rng.integers(0, 40, 500)], 1)
    samples[:20, 1] = samples[:20, 0]                      # same-triangle pairs
    f = S.lag_features(m, problem.ProblemParams(1, 1, 1, 1, 40), samples)
    assert f.shape == (500, S.F)
    assert np.isfinite(f).all() and np.abs(f).max() < 50


def test_labels_smallest_rule_within_tolerance():
    rng = np.random.default_rng(4)
    ref = rng.normal(size=(50, 6))
    blocks = np.stack([ref + rng.normal(scale=s, size=ref.shape) for s in (1e-2, 1e-5, 1e-9)] + [ref])
    lab = S.labels(blocks, 1e-6, 1.0)
    assert (lab == 2).all()
    lab = S.labels(blocks, 1e-3, 1.0)
    assert (lab == 1).all()
    blocks[:, 7] = blocks[3, 7]                            # every rule agrees on sample 7
    assert S.labels(blocks, 0.0, 1.0)[7] == 0
