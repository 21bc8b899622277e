"""Batched form: many instances of uneven size in one graph-captured
schedule chosen by the autotuner (a persistent launch with a tuned tile
shape, or one two-pass assembly per instance), against the binary128
value of the reference's formulas on sampled blocks of every instance (all
lags), and against the single-mesh assembly of each instance (the same
per-pair computation in another kernel) in FP64 and in the mixed-precision
mode, over repeated replays with changing output buffers."""
import numpy as np
import pytest

from conftest import cuda_available

TOL = 1e-12          # FP64: the same per-pair code compiled in two kernels
TOL_MIXED = 1e-6     # mixed precision: FP32 contraction choices differ between the two kernels


@pytest.fixture(scope="module")
def ebem():
    if not cuda_available():
        pytest.skip("no CUDA device")
    import elastodynamicebem_b200.core as core
    return core


@pytest.mark.gpu
@pytest.mark.parametrize("n_gh,prec", [(7, 0), (7, 1), (12, 0)])
def test_batch_equals_single(ebem, n_gh, prec):
    import torch
    from elastodynamicebem_b200 import problem
    inst = problem.batch_workload(count=8, seed=11, n_min=16, n_max=400)
    dms = [ebem.DeviceMesh(m) for _, m, _ in inst]
    prms = [p for _, _, p in inst]
    nlag = [min(ebem.num_blocks(d, p), 12) for d, p in zip(dms, prms)]
    plan = ebem.BatchPlan(dms, prms, n_gh, nlag=nlag, prec=prec)
    singles = [ebem.assemble_sa(d, p, n_gh, 0, l, prec=prec).clone() for d, p, l in zip(dms, prms, nlag)]
    for rep in range(2):
        outs = [torch.full((l, 3 * d.N, 3 * d.N), float("nan"), dtype=torch.float64, device="cuda")
                for d, l in zip(dms, nlag)]
        got = plan.assemble(outs)
        torch.cuda.synchronize()
        for g, s1 in zip(got, singles):
            assert torch.isfinite(g).all()
            assert float((g - s1).norm() / s1.norm()) <= (TOL_MIXED if prec else TOL)
    info = plan.info()
    # 0 / 0: the per-instance schedule won the tuning
    assert (info["warps_per_block"], info["pairs_per_grab"]) in {(w, c) for w in (2, 4) for c in (1, 4, 16)} | {(0, 0)}
    assert info["tuned_ms"] > 0 and info["pairs"] == sum(d.N ** 2 for d in dms)


@pytest.mark.gpu
def test_batch_survives_other_rules_on_its_meshes(ebem):
    """A plan holds device pointers to its meshes' mapped outer nodes; using
    the same meshes with other rules afterwards leaves those tables in place,
    so the plan's next replay gives the same blocks."""
    import torch
    from elastodynamicebem_b200 import problem
    inst = problem.batch_workload(count=4, seed=12, n_min=16, n_max=200)
    dms = [ebem.DeviceMesh(m) for _, m, _ in inst]
    prms = [p for _, _, p in inst]
    nlag = [min(ebem.num_blocks(d, p), 6) for d, p in zip(dms, prms)]
    plan = ebem.BatchPlan(dms, prms, 7, nlag=nlag)
    first = [g.clone() for g in plan.assemble()]
    for d, p in zip(dms, prms):
        for n_gh in (3, 12, 19):
            ebem.assemble_sa(d, p, n_gh, 0, 1)
    outs = [torch.full((l, 3 * d.N, 3 * d.N), float("nan"), dtype=torch.float64, device="cuda")
            for d, l in zip(dms, nlag)]
    again = plan.assemble(outs)
    torch.cuda.synchronize()
    for g, f in zip(again, first):
        assert float((g - f).norm() / f.norm()) <= 1e-14
    plan.close()


@pytest.mark.gpu
@pytest.mark.parametrize("n_gh", [7, 12])
def test_batch_against_exact_blocks(ebem, oracle, n_gh):
    """The batched form at reduced size with all lags of every instance (8
    screens and spheres of uneven size, their own dt and materials), checked
    on a seeded sample of 60 blocks per instance against the binary128 value
    of the reference's formulas (the oracle's "q" evaluation), bar 1e-10; the
    sampled blocks include diagonal ones and the last lags."""
    import os
    import sys
    from conftest import ROOT
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_golden
    from elastodynamicebem_b200 import problem
    inst = problem.batch_workload(count=8, seed=13, n_min=32, n_max=512)
    dms = [ebem.DeviceMesh(m) for _, m, _ in inst]
    prms = [p for _, _, p in inst]
    nlag = [ebem.num_blocks(d, p) for d, p in zip(dms, prms)]          # all lags
    plan = ebem.BatchPlan(dms, prms, n_gh, nlag=nlag)
    got = [g.cpu().numpy() for g in plan.assemble()]
    plan.close()
    for k, ((name, m, p), E, L) in enumerate(zip(inst, got, nlag)):
        src, fld, lag = make_golden.sample(m, p, L, 60, 500 + k)
        exact = oracle.assemble_sa_pairs(m, p, n_gh, src, fld, lag, variant="q")
        blocks = np.stack([E[l, 3 * i:3 * i + 3, 3 * j:3 * j + 3] for i, j, l in zip(src, fld, lag)])
        err = np.linalg.norm(blocks - exact) / np.linalg.norm(exact)
        assert err <= 1e-10, (name, err)
        assert np.isfinite(E).all()


def test_batch_workload_shape():
    from elastodynamicebem_b200 import problem
    inst = problem.batch_workload()
    assert len(inst) == 64
    Ns = [m.numberTriangles for _, m, _ in inst]
    assert min(Ns) >= 128 * 0.7 and max(Ns) <= 2048 * 1.3
    assert all(0.5 <= p.lam <= 3 and 12 <= p.nT <= 50 for _, _, p in inst)
