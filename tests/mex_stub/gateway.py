"""Drives the MEX gateway (elastodynamicebem_b200/mex/ebem_mex.c) without
MATLAB (test infrastructure only): compiles it with gcc against the mex.h
stand-in of this directory and libebem.so, and calls mexFunction with numpy
arrays converted to the stand-in's column-major arrays."""
from __future__ import annotations

import ctypes as C
import os
import shutil
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
PKG = os.path.join(ROOT, "elastodynamicebem_b200")


class MexError(RuntimeError):
    def __init__(self, ident: str, msg: str):
        super().__init__(f"{ident}: {msg}")
        self.ident, self.msg = ident, msg


def build(outdir: str) -> str:
    """Compile gateway + stand-in into outdir/libebem_mex_stub.so."""
    gcc = shutil.which("gcc")
    if gcc is None:
        raise RuntimeError("gcc not available")
    out = os.path.join(outdir, "libebem_mex_stub.so")
    cmd = [gcc, "-std=c99", "-O1", "-Wall", "-Werror", "-Wno-unused-parameter", "-Wno-unused-function", "-fPIC",
           "-shared", "-I", HERE, "-I", os.path.join(ROOT, "include"), "-o", out,
           os.path.join(PKG, "mex", "ebem_mex.c"), os.path.join(HERE, "mex_stub.c"), "-L", PKG, "-lebem",
           f"-Wl,-rpath,{PKG}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return out


class Gateway:
    def __init__(self, path: str):
        # libebem first, so that the gateway binds the same copy the tests use
        from elastodynamicebem_b200 import lib
        lib.load()
        self.L = C.CDLL(path)
        L = self.L
        L.stub_double.restype = C.c_void_p
        L.stub_double.argtypes = [C.c_size_t, C.c_size_t, C.c_size_t, C.c_void_p]
        L.stub_string.restype = C.c_void_p
        L.stub_string.argtypes = [C.c_char_p]
        L.stub_numel.restype = C.c_size_t
        L.stub_numel.argtypes = [C.c_void_p]
        L.stub_dim.restype = C.c_size_t
        L.stub_dim.argtypes = [C.c_void_p, C.c_int]
        L.stub_data.restype = C.POINTER(C.c_double)
        L.stub_data.argtypes = [C.c_void_p]
        L.stub_free.argtypes = [C.c_void_p]
        L.stub_error_id.restype = C.c_char_p
        L.stub_error_msg.restype = C.c_char_p
        L.stub_call.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_void_p]
        L.stub_run_at_exit.restype = C.c_int

    def _arg(self, x):
        if isinstance(x, str):
            return self.L.stub_string(x.encode())
        a = np.asarray(x, dtype=np.float64)
        if a.ndim == 0:
            a = a.reshape(1, 1)
        elif a.ndim == 1:
            a = a.reshape(-1, 1)
        dims = list(a.shape) + [1] * (3 - a.ndim)
        f = np.asfortranarray(a)
        return self.L.stub_double(dims[0], dims[1], dims[2], f.ctypes.data)

    def _out(self, p):
        dims = [self.L.stub_dim(p, k) for k in range(3)]
        n = self.L.stub_numel(p)
        v = np.ctypeslib.as_array(self.L.stub_data(p), shape=(n,)).copy()
        self.L.stub_free(p)
        shape = dims if dims[2] > 1 else dims[:2]
        return v.reshape(shape, order="F")

    def __call__(self, cmd: str, *args, nout: int = 1):
        ins = [self._arg(cmd)] + [self._arg(a) for a in args]
        prhs = (C.c_void_p * len(ins))(*ins)
        plhs = (C.c_void_p * max(1, nout))()
        rc = self.L.stub_call(nout, plhs, len(ins), prhs)
        for p in ins:
            self.L.stub_free(p)
        if rc:
            raise MexError(self.L.stub_error_id().decode(), self.L.stub_error_msg().decode())
        outs = [self._out(plhs[k]) for k in range(nout) if plhs[k]]
        return outs[0] if nout == 1 and outs else outs


def mesh_args(mesh):
    """domainMesh.coordinates and 1-based domainMesh.triangles of a mesh."""
    return np.asarray(mesh.coordinates, np.float64), np.asarray(mesh.triangles, np.float64) + 1


def problem_vec(prm):
    return np.array([prm.rho, prm.mu, prm.lam, prm.Tfin, prm.nT], dtype=np.float64)
