"""The MEX gateway through the mex.h stand-in on the device: every command
family returns what the library's own entry points return, in MATLAB's
layouts (E 3N x 3N x L, density 3N x nT, displacement 3 x npts x ntimes,
1-based triangles in, column-major arrays both ways)."""
import os
import sys

import numpy as np
import pytest

from conftest import ROOT, cuda_available

pytestmark = pytest.mark.gpu
sys.path.insert(0, os.path.join(ROOT, "tests", "mex_stub"))


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def env(tmp_path_factory):
    if not cuda_available():
        pytest.skip("no CUDA device")
    import gateway
    import elastodynamicebem_b200.core as core
    return gateway, gateway.Gateway(gateway.build(str(tmp_path_factory.mktemp("mex")))), core


def test_indirect_commands(env):
    gateway, gw, core = env
    from elastodynamicebem_b200 import mesh, problem
    m, prm = mesh.screen_uniform(4), problem.ProblemParams(1.0, 1.0, 2.0, 1.0, 20)
    P, T, q = *gateway.mesh_args(m), gateway.problem_vec(prm)
    dm = core.DeviceMesh(m)
    L = core.num_blocks(dm, prm)
    assert gw("num_blocks", P, T, q) == L
    E = gw("assemble_sa", P, T, q, 7, 0, L)
    Ed = core.assemble_sa(dm, prm, 7, 0, L).cpu().numpy()          # [l][row, col]
    assert E.shape == (96, 96, L) and np.array_equal(E, Ed.transpose(1, 2, 0))
    b = gw("rhs", P, T, q, 7, 0)
    assert b.shape == (96, 20) and np.array_equal(b, core.rhs(dm, prm, 7, 0).cpu().numpy().T)
    phi = gw("timemarch_sa", P, T, q, 7, 0)
    phid, _ = core.timemarch_sa(dm, prm, 7, 0)
    assert rel(phi, phid.cpu().numpy().T) <= 1e-13
    assert rel(gw("march", E, b), phi) <= 1e-13
    assert rel(gw("timemarch_banded", P, T, q, 7, 0), phi) <= 1e-12
    Eg = gw("assemble_ghc", P, T, q, 7, 16, 3, 0, L)
    assert rel(Eg, core.assemble_ghc(dm, prm, 7, 16, 3, 0, L).cpu().numpy().transpose(1, 2, 0)) <= 1e-15
    phig = gw("timemarch_ghc", P, T, q, 7, 16, 3, 0)
    assert np.isfinite(phig).all() and rel(phig, phi) < 0.2          # numerical inner rule vs closed form
    X = np.array([[0.1, 0.2, 0.31], [-0.3, 0.05, 0.4]])
    t = np.array([0.25, 0.5, 1.0])
    u = gw("pp_sa", P, T, q, phi, X, t)
    ud = core.pp_sa(dm, prm, phid, X, t).cpu().numpy()              # (nt, np, 3)
    assert u.shape == (3, 2, 3) and rel(u, ud.transpose(2, 1, 0)) <= 1e-12
    ug = gw("pp_gpu", P, T, q, phi, X, t, 16, 3, 1)
    assert rel(ug, core.pp_gpu(dm, prm, phid, X, t, 16, 3, 1).cpu().numpy().transpose(2, 1, 0)) <= 1e-12


def test_direct_commands(env):
    gateway, gw, core = env
    import torch
    from elastodynamicebem_b200 import mesh, problem
    m, prm = mesh.prism_bar(1.0, 1.0, 3.0, 0.5), problem.ProblemParams(1.0, 1.0, 2.0, 2.0, 16)
    P, T, q = *gateway.mesh_args(m), gateway.problem_vec(prm)
    rules = np.array([7, 4, 3, 16], dtype=float)
    dm = core.DeviceMesh(m)
    LV, LK = core.num_blocks_dir(dm, prm)
    lv, lk = gw("num_blocks_dir", P, T, q, nout=2)
    assert (int(lv), int(lk)) == (LV, LK)
    V = gw("assemble_v", P, T, q, rules, 0, LV)
    Vd = core.assemble_v(dm, prm, 7, 4, 3, 16, 0, LV).cpu().numpy()
    assert rel(V, Vd.transpose(1, 2, 0)) <= 1e-15
    K = gw("assemble_k", P, T, q, rules, 0, LK)
    Kd = core.assemble_k(dm, prm, 7, 4, 3, 16, 0, LK).cpu().numpy()
    assert K.shape == (3 * m.numberTriangles, 3 * m.number_nodes, LK) and rel(K, Kd.transpose(1, 2, 0)) <= 1e-15
    gV = problem.bar_neumann(m, prm, 3.0)                             # (nT, 3N)
    u = gw("march_dn", P, T, q, rules, gV.T)
    ud = core.march_dn(dm, prm, torch.tensor(Vd, device="cuda"), torch.tensor(Kd, device="cuda"),
                       torch.tensor(gV, device="cuda")).cpu().numpy()
    assert u.shape == (3 * m.number_nodes, prm.nT) and rel(u, ud.T) <= 1e-12
    X = np.array([[0.5, 0.5, 1.5], [0.3, 0.6, 2.2]])
    t = np.array([1.0, 2.0])
    up = gw("pp_dir", P, T, q, 4, 3, gV.T, u, X, t)
    upd = core.pp_dir(dm, prm, 4, 3, torch.tensor(gV, device="cuda"), torch.tensor(u.T.copy(), device="cuda"), X,
                      t).cpu().numpy()
    assert up.shape == (3, 2, 2) and rel(up, upd.transpose(2, 1, 0)) <= 1e-12
