"""Banded storage of the Toeplitz blocks (ebem_banded_*): the blocks equal the
dense assembly's, the non-null count equals its count, and the marching on
the bands equals the dense marching; sizes and times of both are printed."""
import pytest

from conftest import cuda_available

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ebem():
    if not cuda_available():
        pytest.skip("no CUDA device")
    import elastodynamicebem_b200.core as core
    return core


def rel(a, b):
    return float((a - b).norm() / b.norm())


@pytest.mark.parametrize("case", ["screen128", "sphere320"])
def test_banded_equals_dense(ebem, case):
    from elastodynamicebem_b200 import problem
    w = problem.screen_workload() if case == "screen128" else problem.sphere_workload(7, 2)
    dm = ebem.DeviceMesh(w.mesh)
    L = ebem.num_blocks(dm, w.params)
    E, cnt = ebem.assemble_sa(dm, w.params, w.n_gh, 0, L, count=True)
    B = ebem.BandedOperator(dm, w.params, w.n_gh)
    info = B.info()
    assert info["L"] == L and info["nonnull"] == cnt
    assert info["bytes"] < 8 * (3 * dm.N) ** 2 * L
    Eb = B.to_dense()
    # the banded blocks come from the one-warp-per-pair kernel, the dense ones
    # from the two-pass level kernel: the same terms summed in another order
    assert rel(Eb, E) <= 1e-14
    part = B.to_dense(3, 5)
    assert bool((part == Eb[3:8]).all())
    b = ebem.rhs(dm, w.params, w.n_gh, w.datum)
    phi = ebem.march(E, b)
    assert rel(B.march(b), phi) <= 1e-12
    Bm = ebem.BandedOperator(dm, w.params, w.n_gh, prec=ebem.PREC_MIXED)
    Em = ebem.assemble_sa(dm, w.params, w.n_gh, 0, L, prec=ebem.PREC_MIXED)
    # FP32 partial sums grouped differently by the two kernels: within the
    # mixed form's own error scale (1.9e-6 against FP64 on the sphere)
    assert rel(Bm.to_dense(), Em) <= 1e-6
    B.close()
    Bm.close()


def test_banded_sphere1280_memory_and_time(ebem):
    import torch
    from elastodynamicebem_b200 import problem
    w = problem.sphere_workload(7)
    dm = ebem.DeviceMesh(w.mesh)
    L = ebem.num_blocks(dm, w.params)
    b = ebem.rhs(dm, w.params, w.n_gh, w.datum)

    def timed(fn):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        out = fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), out

    ta, E = timed(lambda: ebem.assemble_sa(dm, w.params, w.n_gh, 0, L))
    tm, phi = timed(lambda: ebem.march(E, b))
    dense_bytes = E.numel() * 8
    del E
    torch.cuda.empty_cache()
    tb, B = timed(lambda: ebem.BandedOperator(dm, w.params, w.n_gh))
    tbm, phib = timed(lambda: B.march(b))
    info = B.info()
    print(f"\nsphere N={dm.N} L={L}: dense {dense_bytes / 1e9:.2f} GB, assembly {ta:.1f} ms, march {tm:.1f} ms; "
          f"banded {info['bytes'] / 1e9:.2f} GB, assembly {tb:.1f} ms, march {tbm:.1f} ms")
    assert rel(phib, phi) <= 1e-12
    assert info["bytes"] < dense_bytes / 3
