"""Device-side mesh fields and the library's state across a device reset.

* ebem_mesh_derived against the derived fields of the reference's mesh
  reader (f/utility/fileRead/readSpaceMesh.m:114-139), restated here in numpy:
  n = (P1 - P3) x (P2 - P3) / |.|, area = |.| / 2, centroid, longest edge.
* ebem_device_release before a cudaDeviceReset (the reference's GPU marching
  resets the device at entry and exit, BEMenerg_coreGPU_timeMarching.m:7,170):
  a child process runs the assembly, the allocation-free assembly and the
  marching, releases the library's state, resets the device and runs them
  again; the assemblies must be identical bit for bit, the marching equal to
  rounding (its history sum adds with atomics).
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT, cuda_available

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def core():
    if not cuda_available():
        pytest.skip("no CUDA device")
    import elastodynamicebem_b200.core as c
    return c


def read_space_mesh_fields(coords, tris):
    """readSpaceMesh.m:93-139 restated (triangles 0-based)."""
    P1, P2, P3 = coords[tris[:, 0]], coords[tris[:, 1]], coords[tris[:, 2]]
    vg1, vg2, vg3 = P1 - P3, P2 - P3, P1 - P2
    n = np.stack([vg1[:, 1] * vg2[:, 2] - vg2[:, 1] * vg1[:, 2],
                  -vg1[:, 0] * vg2[:, 2] + vg2[:, 0] * vg1[:, 2],
                  vg1[:, 0] * vg2[:, 1] - vg2[:, 0] * vg1[:, 1]], axis=1)
    area = np.sqrt((n ** 2).sum(1)) / 2
    normal = n / (2 * area)[:, None]
    center = (P1 + P2 + P3) / 3
    lens = np.stack([np.sqrt((vg3 ** 2).sum(1)), np.sqrt((vg2 ** 2).sum(1)), np.sqrt((vg1 ** 2).sum(1))], axis=1)
    return normal, area, center, lens.max(1)


@pytest.mark.parametrize("name", ["screen", "sphere", "prism", "graded"])
def test_mesh_derived_fields(core, name):
    from elastodynamicebem_b200 import mesh
    m = {"screen": lambda: mesh.screen_uniform(8), "sphere": lambda: mesh.icosphere(3),
         "prism": lambda: mesh.prism_bar(1.0, 1.0, 3.0, 0.25), "graded": lambda: mesh.screen_graded(6, 4)}[name]()
    dm = core.DeviceMesh(m)
    n, a, c, ml = dm.derived()
    rn, ra, rc, rm = read_space_mesh_fields(np.asarray(m.coordinates, float), np.asarray(m.triangles))
    for got, want in ((n, rn), (a, ra), (c, rc), (ml, rm)):
        assert np.allclose(got, want, rtol=1e-14, atol=1e-15)
    # the host-side fields of the mesh object (used by the oracle) agree as well
    assert np.allclose(m.area, ra, rtol=1e-14) and np.allclose(m.maxL, rm, rtol=1e-14)


CHILD = r"""
import ctypes as C, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from elastodynamicebem_b200 import lib as Lb, mesh, problem
L = Lb.load()
cudart = C.CDLL("libcudart.so.12")
m, prm = mesh.screen_uniform(4), problem.ProblemParams(1.0, 1.0, 2.0, 1.0, 20)

def run():
    h = C.c_void_p()
    coords = np.ascontiguousarray(m.coordinates, np.float64)
    tris = np.ascontiguousarray(m.triangles, np.int32)
    Lb.check(L.ebem_mesh_create(coords.ctypes.data, m.number_nodes, tris.ctypes.data, m.numberTriangles, C.byref(h)))
    p = Lb.problem_struct(prm)
    nb = C.c_int()
    Lb.check(L.ebem_num_blocks(h, C.byref(p), C.byref(nb)))
    n3 = 3 * m.numberTriangles
    E = np.zeros(n3 * n3 * nb.value)
    Lb.check(L.ebem_assemble_sa(h, C.byref(p), 7, 0, nb.value, E.ctypes.data, 0, None, None))
    rhs = np.zeros(n3 * prm.nT)
    Lb.check(L.ebem_rhs(h, C.byref(p), 7, 0, rhs.ctypes.data, None))
    phi = np.zeros(n3 * prm.nT)
    Lb.check(L.ebem_march(E.ctypes.data, n3, nb.value, rhs.ctypes.data, prm.nT, phi.ctypes.data, None))
    d = C.c_void_p()
    assert cudart.cudaMalloc(C.byref(d), C.c_size_t(E.nbytes)) == 0
    Lb.check(L.ebem_assemble_sa_noalloc(h, C.byref(p), 7, 0, nb.value, d, 0, None, None))
    Ena = np.zeros_like(E)
    assert cudart.cudaMemcpy(C.c_void_p(Ena.ctypes.data), d, C.c_size_t(E.nbytes), 2) == 0   # device to host
    cudart.cudaFree(d)
    Lb.check(L.ebem_mesh_destroy(h))
    return E, phi, Ena

a = run()
Lb.check(L.ebem_device_release(0))
assert cudart.cudaDeviceReset() == 0
b = run()
rel = lambda x, y: np.linalg.norm(x - y) / np.linalg.norm(y)
assert np.array_equal(a[0], b[0]) and np.array_equal(a[2], b[2])    # the assemblies are deterministic
assert rel(b[1], a[1]) <= 1e-13                                     # the marching's history sum adds with atomics
assert rel(a[2], a[0]) <= 1e-14
assert np.isfinite(a[1]).all() and np.abs(a[1]).max() > 0
print("reset-ok")
"""


def test_release_then_device_reset(core):
    env = dict(os.environ, CUDA_VISIBLE_DEVICES=os.environ.get("CUDA_VISIBLE_DEVICES", "0").split(",")[0])
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT], capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0 and "reset-ok" in r.stdout, r.stdout + r.stderr
