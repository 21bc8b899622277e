"""The MEX gateway (elastodynamicebem_b200/mex/ebem_mex.c) compiled with gcc
against a stand-in for MATLAB's mex.h (tests/mex_stub) and called through it
on the CPU: it builds with -Wall -Werror, host-only commands return the
library's values in MATLAB's layouts, every library error becomes a MATLAB
error (mexErrMsgIdAndTxt) with the library's message, and compute commands
fail cleanly without a device (no CPU path)."""
import os
import sys

import numpy as np
import pytest

from conftest import ROOT, cuda_available

sys.path.insert(0, os.path.join(ROOT, "tests", "mex_stub"))


@pytest.fixture(scope="module")
def gw(tmp_path_factory):
    import gateway
    return gateway.Gateway(gateway.build(str(tmp_path_factory.mktemp("mex"))))


def test_version_and_quadrature(gw):
    from elastodynamicebem_b200 import core
    assert gw("version") == 1
    n, w = gw("quad_gh", 7, 4, nout=2)
    rn, rw = core.quad_gh(7, 4)
    assert n.shape == (28, 3) and np.array_equal(n, rn)          # MATLAB's (nSub nNodes) x 3
    assert np.array_equal(w.ravel(), rw)


def test_errors_become_matlab_errors(gw):
    import gateway
    with pytest.raises(gateway.MexError) as ei:
        gw("quad_gh", 5, 1)
    assert ei.value.ident == "ebem:quad_gh" and "Gauss-Hammer" in ei.value.msg
    with pytest.raises(gateway.MexError) as ei:
        gw("no_such_command")
    assert "unknown command" in ei.value.msg
    with pytest.raises(gateway.MexError) as ei:
        gw("assemble_sa", np.zeros((3, 3)))
    assert "usage" in ei.value.msg
    with pytest.raises(gateway.MexError) as ei:
        gw("march", np.zeros((6, 6, 2)), np.zeros((5, 4)))
    assert "do not match" in ei.value.msg


@pytest.mark.skipif(cuda_available(), reason="checks the no-device error path")
def test_compute_commands_need_a_device(gw):
    import gateway
    from elastodynamicebem_b200 import mesh, problem
    m, prm = mesh.screen_uniform(2), problem.ProblemParams(1.0, 1.0, 2.0, 1.0, 4)
    P, T = gateway.mesh_args(m)
    for cmd, extra in (("assemble_sa", (7, 0, 2)), ("num_blocks", ()), ("timemarch_sa", (7, 0))):
        with pytest.raises(gateway.MexError) as ei:
            gw(cmd, P, T, gateway.problem_vec(prm), *extra)
        assert "no CUDA device" in ei.value.msg


def test_release_and_exit_hook(gw):
    gw("release")
    assert gw.L.stub_run_at_exit() == 1          # the gateway registered its exit hook
