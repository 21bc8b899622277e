"""Build libebem.so in-tree with nvcc for sm_100a.

The library is plain CUDA C++ behind the C ABI of include/ebem.h; Python
loads it with ctypes (no torch types cross the boundary).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libebem.so")

SOURCES = ["capi.cu", "quadrature.cu", "sa_assemble.cu", "march.cu", "ghc.cu", "direct.cu", "selector.cu", "banded.cu", "pp_num.cu", "sa_twopass.cu"]
HEADERS = ["sa_device.cuh", "sa_edge.cuh", "sa_pair.cuh", "sa_warp.cuh", "ebem_internal.h", "ptr_kind.h"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
         "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include")]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(ROOT, "include", "ebem.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False,
          defines: tuple = (), out: str | None = None) -> str:
    """Compile and link libebem.so.  ``defines`` adds -D flags and ``out``
    redirects the library (used to compare code-generation options)."""
    target = out or LIB
    if not force and out is None and not _stale():
        return LIB
    objdir = os.path.join(PKG, "_build" if out is None else "_build_" + os.path.basename(out).replace(".so", ""))
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for src in SOURCES:
        obj = os.path.join(objdir, src.replace(".cu", ".o"))
        cmd = [nvcc(), *ARCH, *FLAGS, *[f"-D{d}" for d in defines], "-c", os.path.join(CSRC, src), "-o", obj]
        if ptxas_info:
            cmd += ["-Xptxas", "-v"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stderr}")
        if ptxas_info or verbose:
            print(r.stderr, file=sys.stderr)
        objs.append(obj)
    tmp = target + ".tmp"
    cmd = [nvcc(), *ARCH, "-shared", "-o", tmp, *objs, "-lcudart", "-lcusolver", "-lcublas"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr}")
    os.replace(tmp, target)
    return target


if __name__ == "__main__":
    build(force=True, verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
