"""The marching pieces of the C ABI on the device (ebem_lu_*,
ebem_history_gemv) and the row-panel marching of shard.march_panels on one
rank against ebem_march."""
import numpy as np
import pytest

from conftest import cuda_available

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ebem():
    if not cuda_available():
        pytest.skip("no CUDA device")
    import elastodynamicebem_b200.core as core
    return core


def test_lu_and_history_gemv(ebem):
    import torch
    g = torch.Generator(device="cuda").manual_seed(3)
    n = 300
    A = torch.randn((n, n), dtype=torch.float64, device="cuda", generator=g) + n * torch.eye(n, dtype=torch.float64,
                                                                                             device="cuda")
    b = torch.randn((2, n), dtype=torch.float64, device="cuda", generator=g)
    lu = ebem.DeviceLU(A)
    x = lu.solve(b.clone())
    assert float((x @ A.t() - b).norm() / b.norm()) <= 1e-13
    rows, K = 77, 1000
    M = torch.randn((K, rows), dtype=torch.float64, device="cuda", generator=g)      # column-major rows x K
    v = torch.randn(K, dtype=torch.float64, device="cuda", generator=g)
    y0 = torch.randn(rows, dtype=torch.float64, device="cuda", generator=g)
    y = ebem.history_gemv(M, rows, v, y0.clone())
    assert float((y - (y0 - M.t() @ v)).norm() / y0.norm()) <= 1e-13
    Z = torch.zeros((n, n), dtype=torch.float64, device="cuda")
    from elastodynamicebem_b200.lib import EbemError
    with pytest.raises(EbemError):
        ebem.DeviceLU(Z)


def test_panel_marching_single_rank(ebem):
    from elastodynamicebem_b200 import problem, shard
    w = problem.sphere_workload(7, 2)
    dm = ebem.DeviceMesh(w.mesh)
    L = ebem.num_blocks(dm, w.params)
    N = dm.N
    panel = ebem.assemble_sa_panel(dm, w.params, w.n_gh, 0, L, 0, N)
    b = ebem.rhs(dm, w.params, w.n_gh, w.datum)
    phi = shard.march_panels(panel, b, N, 1, 0)
    E = panel.view(L, 3 * N, 3 * N).transpose(1, 2)
    ref = ebem.march(E, b)
    assert float((phi - ref).norm() / ref.norm()) <= 1e-12
