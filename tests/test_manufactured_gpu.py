"""The reference's manufactured case 'TEST' on the device: the right-hand side
(datum 8, closed-form radial integrals) against the oracle's cubature, and the
known answer phi = (1, 1, 1) of the semi-analytic path end to end (assembly,
right-hand side, marching) in FP64 and in the mixed-precision form."""
import os
import sys

import numpy as np
import pytest

from conftest import cuda_available

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import oracle as O  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ebem():
    if not cuda_available():
        pytest.skip("no CUDA device")
    import elastodynamicebem_b200.core as core
    return core


def test_rhs_test_matches_oracle(ebem):
    from elastodynamicebem_b200 import mesh, problem
    m, prm = mesh.screen_uniform(4, half=1.0), problem.ProblemParams(1.0, 1.0, 2.0, 1.0, 10)
    dm = ebem.DeviceMesh(m)
    b = ebem.rhs(dm, prm, 7, problem.DATUM_TEST).cpu().numpy()
    bo = O.rhs(m, prm, 7, problem.DATUM_TEST)
    assert np.linalg.norm(b.T - bo) <= 1e-12 * np.linalg.norm(bo)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_known_answer(ebem, prec):
    from elastodynamicebem_b200 import mesh, problem
    m, prm = mesh.screen_uniform(8, half=1.0), problem.ProblemParams(1.0, 1.0, 2.0, 1.0, 20)
    dm = ebem.DeviceMesh(m)
    p = ebem.PREC_FP64 if prec == "fp64" else ebem.PREC_MIXED
    phi, L = ebem.timemarch_sa(dm, prm, 7, problem.DATUM_TEST, prec=p)
    err = float((phi - 1).abs().max())
    print(f"\nTEST screen N={m.numberTriangles}, L={L}, {prec}: max |phi - 1| = {err:.2e}")
    assert err <= (1e-11 if prec == "fp64" else 1e-6)


def test_test_datum_rejects_other_meshes(ebem):
    import torch
    from elastodynamicebem_b200 import lib, mesh, problem
    for m in (mesh.screen_uniform(4), mesh.icosphere(1)):       # [-0.5,0.5]^2 passes the box test; the sphere not
        dm = ebem.DeviceMesh(m)
        out = torch.empty(3 * m.numberTriangles * 4, dtype=torch.float64, device="cuda")
        prm = problem.ProblemParams(1.0, 1.0, 2.0, 1.0, 4)
        import ctypes as C
        rc = lib.load().ebem_rhs(dm.handle, C.byref(lib.problem_struct(prm)), 7, 8, out.data_ptr(), None)
        assert rc == (0 if m.numberTriangles == 32 else -1)
