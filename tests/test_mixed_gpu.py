"""Mixed-precision form of the semi-analytic assembly (FP32 bulk quadrature,
FP64 closed-form pieces at the fronts and the singularity, FP64 level
combination, factorisation and time marching) against the FP64 path:
the error of the blocks, of the time-marched density and of the
post-processed displacement."""
import numpy as np
import pytest

from conftest import cuda_available

pytestmark = pytest.mark.gpu

TOL_E = 1e-5          # assembled blocks, all lags (Frobenius, relative)
TOL_FIELD = 1e-6      # time-marched density and displacement (Frobenius over all steps / points x times)


@pytest.fixture(scope="module")
def ebem():
    if not cuda_available():
        pytest.skip("no CUDA device")
    import elastodynamicebem_b200.core as core
    return core


def rel(a, b):
    return float((a - b).norm() / b.norm())


@pytest.mark.parametrize("case", ["screen128", "sphere320"])
def test_mixed_against_fp64(ebem, case):
    from elastodynamicebem_b200 import problem
    w = problem.screen_workload() if case == "screen128" else problem.sphere_workload(7, 2)
    dm = ebem.DeviceMesh(w.mesh)
    L = ebem.num_blocks(dm, w.params)
    E64 = ebem.assemble_sa(dm, w.params, w.n_gh, 0, L).clone()
    E32 = ebem.assemble_sa(dm, w.params, w.n_gh, 0, L, prec=ebem.PREC_MIXED)
    assert rel(E32, E64) <= TOL_E
    phi64, _ = ebem.timemarch_sa(dm, w.params, w.n_gh, w.datum)
    phi32, _ = ebem.timemarch_sa(dm, w.params, w.n_gh, w.datum, prec=ebem.PREC_MIXED)
    assert rel(phi32, phi64) <= TOL_FIELD
    u64 = ebem.pp_sa(dm, w.params, phi64, w.points[:64], w.times)
    u32 = ebem.pp_sa(dm, w.params, phi32, w.points[:64], w.times)
    assert rel(u32, u64) <= TOL_FIELD


def test_mixed_rejects_unknown_mode(ebem):
    import ctypes as C
    from elastodynamicebem_b200 import lib, mesh, problem
    m, prm = mesh.screen_uniform(2), problem.ProblemParams(1, 1, 2, 1, 4)
    dm = ebem.DeviceMesh(m)
    import torch
    out = torch.empty(9 * m.numberTriangles ** 2, dtype=torch.float64, device="cuda")
    p = lib.problem_struct(prm)
    rc = lib.load().ebem_assemble_sa_ex(dm.handle, C.byref(p), 7, 0, 1, 0, dm.N, out.data_ptr(), 3 * dm.N, 0, 7,
                                        None, None)
    assert rc == -1
