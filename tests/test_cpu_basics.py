"""CPU-side checks: the C-ABI library loads and exports every entry point of
include/ebem.h, host-only entry points agree with the oracle bit for bit, the
quadrature tables are exact to their degree, and compute entry points refuse
to run without a device (no CPU fallback)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT, cuda_available

HEADER = os.path.join(ROOT, "include", "ebem.h")


def header_symbols():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ebem_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    from elastodynamicebem_b200 import lib as L
    return L.load()


def test_library_exports_header_symbols(lib):
    syms = header_symbols()
    assert len(syms) >= 8
    for s in syms:
        assert hasattr(lib, s), f"libebem.so does not export {s}"
    from elastodynamicebem_b200 import lib as L
    assert set(syms) <= set(L.PROTOTYPES), "ctypes prototypes missing for some header symbols"
    assert lib.ebem_version() == 1


@pytest.mark.parametrize("n", [1, 3, 7, 12, 19, 28])
@pytest.mark.parametrize("nsub", [1, 4, 16, 64])
def test_quad_matches_oracle(lib, oracle, n, nsub):
    from elastodynamicebem_b200 import core
    nodes, w = core.quad_gh(n, nsub)
    on, ow = oracle.gauss_hammer(n, nsub)
    assert np.array_equal(nodes, on) and np.array_equal(w, ow)
    assert abs(w.sum() * nsub - 1.0) < 1e-12


@pytest.mark.parametrize("n,deg", [(1, 1), (3, 2), (7, 5), (12, 6), (19, 9), (28, 11)])
def test_quad_exactness(n, deg):
    """Integrate x^a y^b over the reference triangle (area 1/2) exactly."""
    from math import factorial
    from elastodynamicebem_b200 import core
    for nsub in (1, 4):
        nodes, w = core.quad_gh(n, nsub)
        W = np.tile(w, nsub) / nsub * 0.5 * nsub / 1.0   # composite weights sum to 1 -> area 1/2
        W = np.tile(w, nsub) * 0.5
        x, y = nodes[:, 0], nodes[:, 1]
        tol = 1e-12 if n != 7 else 1e-11     # the 7-point table carries 13 digits
        for a in range(deg + 1):
            for b in range(deg + 1 - a):
                exact = factorial(a) * factorial(b) / factorial(a + b + 2)
                got = (W * x ** a * y ** b).sum()
                assert abs(got - exact) <= tol, (n, nsub, a, b, got, exact)


def test_invalid_rule_rejected(lib):
    from elastodynamicebem_b200 import lib as L
    out = np.zeros(100)
    rc = lib.ebem_quad_gh(5, 1, out.ctypes.data, out.ctypes.data)
    assert rc == -1 and b"Gauss-Hammer" in lib.ebem_last_error()
    rc = lib.ebem_quad_gh(7, 3, out.ctypes.data, out.ctypes.data)
    assert rc == -1


@pytest.mark.skipif(cuda_available(), reason="checks the no-device error path")
def test_no_device_no_fallback(lib):
    from elastodynamicebem_b200 import mesh as M, core
    from elastodynamicebem_b200.lib import EbemError
    with pytest.raises(EbemError) as ei:
        core.DeviceMesh(M.screen_uniform(2))
    assert ei.value.code == -4


def test_mesh_validation(lib):
    coords = np.zeros((3, 3))
    tris = np.array([[0, 1, 5]], np.int32)
    h = C.c_void_p()
    rc = lib.ebem_mesh_create(coords.ctypes.data, 3, tris.ctypes.data, 1, C.byref(h))
    assert rc == -1 and b"out of range" in lib.ebem_last_error()


def test_argument_checks_before_any_device_use(lib):
    """Calls with missing arguments fail with EBEM_ERR_INVALID and a message
    before touching a device, and releasing the workspace when no pool was
    ever created succeeds (all of it runs without a GPU)."""
    out = C.c_void_p()
    assert lib.ebem_release_workspace() == 0
    assert lib.ebem_lu_create(None, 4, None, C.byref(out)) == -1 and not out.value
    assert b"bad arguments" in lib.ebem_last_error()
    assert lib.ebem_lu_solve(None, None, 1, None) == -1
    assert lib.ebem_pp_sa(None, None, None, None, 1, None, 1, None, None) == -1
    assert lib.ebem_march(None, 3, 1, None, 1, None, None) == -1
    assert lib.ebem_batch_create(None, None, None, 0, 7, 0, C.byref(out)) == -1
    # the selector's entry points and the composite-rule blocks
    assert lib.ebem_sa_pair_blocks(None, None, 7, 4, None, 8, 3, None, None) == -1
    assert lib.ebem_selector_sweeps(None, None, None, 8, None, None) == -1
    assert lib.ebem_selector_labels(None, -1, 1e-10, 1.0, None, None, None) == -1
    assert lib.ebem_selector_labels(None, 8, 1e-10, 1.0, None, None, None) == -1
    assert lib.ebem_selector_infer(None, None, None, 0.9, 0, 4, None, None, None) == -1
    assert lib.ebem_assemble_sa_selected(None, None, None, 4, None, 0, 4, None, 0, None, None) == -1
    assert lib.ebem_selector_labels(None, 0, 1e-10, 1.0, None, None, None) == 0      # nothing to label


def test_device_state_release_without_device(lib):
    """ebem_device_release and ebem_workspace_info on a device the library has
    never used: nothing is cached, both succeed without touching a GPU; an
    ordinal outside the supported range is refused."""
    r, u = C.c_ulonglong(7), C.c_ulonglong(7)
    assert lib.ebem_workspace_info(0, C.byref(r), C.byref(u)) == 0
    assert (r.value, u.value) == (0, 0)
    assert lib.ebem_device_release(0) == 0
    assert lib.ebem_device_release(-1) == -1 and b"out of range" in lib.ebem_last_error()
    assert lib.ebem_device_release(64) == -1
    assert lib.ebem_workspace_info(64, None, None) == -1


def test_pointer_classification(tmp_path):
    """The C ABI's buffer classification (csrc/ptr_kind.h): device memory of
    the call's device is used in place, device memory of another GPU is
    refused, managed memory is usable from every device, host memory (pinned
    or not) is staged.  Compiled with g++ and run on the CPU."""
    import shutil
    import subprocess
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    src = tmp_path / "ptr_kind_check.cpp"
    src.write_text(r'''
#include "ptr_kind.h"
#include <cstdio>
using ebem::PtrKind;
using ebem::classify_pointer;
int main() {
    int bad = 0;
    // (cudaMemoryType, owning device, current device) -> kind
    struct { int t, owner, cur; PtrKind want; } cases[] = {
        {0, -2, 0, PtrKind::Host},  {1, 0, 0, PtrKind::Host},   {1, 1, 0, PtrKind::Host},
        {2, 0, 0, PtrKind::Device}, {2, 3, 3, PtrKind::Device}, {2, 1, 0, PtrKind::OtherDevice},
        {2, 0, 5, PtrKind::OtherDevice}, {3, 0, 0, PtrKind::Device}, {3, 2, 0, PtrKind::Device},
    };
    for (auto& c : cases)
        if (classify_pointer(c.t, c.owner, c.cur) != c.want) { std::printf("case %d %d %d\n", c.t, c.owner, c.cur); bad++; }
    return bad;
}
''')
    exe = tmp_path / "ptr_kind_check"
    subprocess.run([gxx, "-std=c++17", "-I", os.path.join(ROOT, "elastodynamicebem_b200", "csrc"), str(src), "-o",
                    str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout
