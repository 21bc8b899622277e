"""The allocation-free assembly entry point, ebem_assemble_sa_noalloc.

Some callers may not allocate device memory while they run: code inside a
host framework that hands out all device memory from its own pool, or a
time-critical loop where a cudaMalloc/cudaFree (which can synchronise the
device) is not allowed.  For them the library keeps the assembly's own small
buffers (mapped outer nodes, non-null counter) in one static 1 MiB device
array.  These tests call it through the C ABI and check it against the
ordinary entry point, ebem_assemble_sa, on consecutive calls (the second call
reuses the array the first one left behind).  This file is collected last.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import cuda_available

pytestmark = pytest.mark.gpu

TOL = 1e-10


@pytest.fixture(scope="module")
def env():
    if not cuda_available():
        pytest.skip("no CUDA device")
    import torch
    from elastodynamicebem_b200 import core, lib
    return torch, core, lib, lib.load()


def _ordinary(env, dm, prm, n_gh, nlag):
    torch, core, lib, L = env
    n3 = 3 * dm.N
    out = torch.empty(nlag * n3 * n3, dtype=torch.float64, device="cuda")
    p = lib.problem_struct(prm)
    cnt = C.c_longlong(-1)
    lib.check(L.ebem_assemble_sa(dm.handle, C.byref(p), n_gh, 0, nlag, C.c_void_p(out.data_ptr()), 0, None,
                                 C.byref(cnt)))
    torch.cuda.synchronize()
    return out, cnt.value


def _noalloc(env, dm, prm, n_gh, nlag):
    torch, core, lib, L = env
    n3 = 3 * dm.N
    out = torch.full((nlag * n3 * n3,), float("nan"), dtype=torch.float64, device="cuda")
    p = lib.problem_struct(prm)
    cnt = C.c_longlong(-1)
    rc = L.ebem_assemble_sa_noalloc(dm.handle, C.byref(p), n_gh, 0, nlag, C.c_void_p(out.data_ptr()), 0, None,
                                    C.byref(cnt))
    assert rc == 0, L.ebem_last_error()
    torch.cuda.synchronize()
    return out, cnt.value


def _rel(a, b):
    return float((a - b).norm() / b.norm())


@pytest.mark.parametrize("case", ["screen128_gh7", "sphere320_gh12"])
def test_matches_ordinary_assembly_twice(env, case):
    torch, core, lib, L = env
    from elastodynamicebem_b200 import problem
    if case == "screen128_gh7":
        w, n_gh = problem.screen_workload(), 7
    else:
        w, n_gh = problem.sphere_workload(12, 2), 12
    dm = core.DeviceMesh(w.mesh)
    nlag = core.num_blocks(dm, w.params)
    ref, cref = _ordinary(env, dm, w.params, n_gh, nlag)
    for _ in range(2):                        # two calls in a row share the scratch array
        got, c = _noalloc(env, dm, w.params, n_gh, nlag)
        assert torch.isfinite(got).all()
        assert _rel(got, ref) <= TOL
        assert c == cref


def test_rule_change_between_calls(env):
    """A call with another outer rule rewrites the shared node table; the next
    call with the first rule must not see stale nodes."""
    torch, core, lib, L = env
    from elastodynamicebem_b200 import mesh, problem
    m, prm = mesh.screen_uniform(4), problem.ProblemParams(1.0, 1.0, 2.0, 1.0, 20)
    dm = core.DeviceMesh(m)
    nlag = core.num_blocks(dm, prm)
    ref7, _ = _ordinary(env, dm, prm, 7, nlag)
    ref3, _ = _ordinary(env, dm, prm, 3, nlag)
    a, _ = _noalloc(env, dm, prm, 3, nlag)
    b, _ = _noalloc(env, dm, prm, 7, nlag)
    assert _rel(a, ref3) <= TOL and _rel(b, ref7) <= TOL


def test_allocates_nothing(env):
    """What the entry point exists for: with the library's workspace pool
    emptied and a fresh mesh handle (no cached outer-node table), two calls
    in a row leave the pool empty, build no table in the mesh and take no
    device memory (free bytes unchanged), and still match the ordinary
    assembly, which does allocate (it builds and caches the table)."""
    torch, core, lib, L = env
    from elastodynamicebem_b200 import problem
    w = problem.screen_workload()
    dm = core.DeviceMesh(w.mesh)
    nlag = core.num_blocks(dm, w.params)
    n3 = 3 * dm.N
    out = torch.empty(nlag * n3 * n3, dtype=torch.float64, device="cuda")
    p = lib.problem_struct(w.params)
    dev = torch.cuda.current_device()

    def state():
        mask, nbytes = C.c_int(-1), C.c_longlong(-1)
        lib.check(L.ebem_mesh_cache_info(dm.handle, C.byref(mask), C.byref(nbytes)))
        res, used = C.c_ulonglong(), C.c_ulonglong()
        lib.check(L.ebem_workspace_info(dev, C.byref(res), C.byref(used)))
        return mask.value, nbytes.value, res.value, used.value

    lib.check(L.ebem_assemble_sa_noalloc(dm.handle, C.byref(p), 7, 0, nlag, C.c_void_p(out.data_ptr()), 0, None,
                                         None))                     # first call: one-time address look-up
    torch.cuda.synchronize()
    lib.check(L.ebem_release_workspace())
    before = state()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(2):
        lib.check(L.ebem_assemble_sa_noalloc(dm.handle, C.byref(p), 7, 0, nlag, C.c_void_p(out.data_ptr()), 0,
                                             None, None))
    torch.cuda.synchronize()
    after = state()
    assert torch.cuda.mem_get_info()[0] == free0
    assert after == before
    assert before[0] == 0 and before[2] == 0 and before[3] == 0    # no table cached, pool empty
    got = out.clone()
    ref, _ = _ordinary(env, dm, w.params, 7, nlag)
    assert _rel(got, ref) <= TOL
    mask, nbytes, _, _ = state()
    assert mask == 1 << 2 and nbytes > after[1]          # the ordinary call cached the 7-node table


def test_count_refused_under_capture(env):
    """The non-null count is read back and waited for, which a stream under
    capture does not allow: such a call is refused before it does any work."""
    torch, core, lib, L = env
    from elastodynamicebem_b200 import mesh, problem
    m, prm = mesh.screen_uniform(2), problem.ProblemParams(1.0, 1.0, 2.0, 1.0, 4)
    dm = core.DeviceMesh(m)
    out = torch.zeros(9 * m.numberTriangles ** 2, dtype=torch.float64, device="cuda")
    p = lib.problem_struct(prm)
    cnt = C.c_longlong(-1)
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        g.capture_begin()
        rc = L.ebem_assemble_sa_noalloc(dm.handle, C.byref(p), 7, 0, 1, C.c_void_p(out.data_ptr()), 0,
                                        C.c_void_p(s.cuda_stream), C.byref(cnt))
        msg = L.ebem_last_error()
        g.capture_end()
    assert rc == -1 and b"capture" in msg and cnt.value == -1


def test_rejects_mesh_beyond_scratch(env):
    torch, core, lib, L = env
    from elastodynamicebem_b200 import mesh, problem
    m, prm = mesh.screen_uniform(64), problem.ProblemParams(1.0, 1.0, 2.0, 1.0, 20)   # 8192 triangles
    dm = core.DeviceMesh(m)
    out = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = lib.problem_struct(prm)
    rc = L.ebem_assemble_sa_noalloc(dm.handle, C.byref(p), 7, 0, 1, C.c_void_p(out.data_ptr()), 0, None, None)
    assert rc == -1
    assert b"too large" in L.ebem_last_error()


def test_rejects_host_output(env):
    torch, core, lib, L = env
    from elastodynamicebem_b200 import mesh, problem
    m, prm = mesh.screen_uniform(2), problem.ProblemParams(1.0, 1.0, 2.0, 1.0, 4)
    dm = core.DeviceMesh(m)
    host = np.zeros(9 * m.numberTriangles ** 2)
    p = lib.problem_struct(prm)
    rc = L.ebem_assemble_sa_noalloc(dm.handle, C.byref(p), 7, 0, 1, C.c_void_p(host.ctypes.data), 0, None, None)
    assert rc == -1
