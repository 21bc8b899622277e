"""ctypes binding of libebem.so (the C ABI of include/ebem.h).

The shared library is built in-tree (``elastodynamicebem_b200/libebem.so``)
by ``build.py``.  Loading fails loudly when the library is missing; there is
no Python or CPU fallback for any compute entry point.
"""
from __future__ import annotations

import ctypes as C
import os

from . import build as _build

_LIB = None


class EbemError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"libebem error {code}: {msg}")
        self.code = code


class ProblemC(C.Structure):
    _fields_ = [("rho", C.c_double), ("mu", C.c_double), ("lambda_", C.c_double),
                ("tfin", C.c_double), ("nt", C.c_int)]


# name -> (restype, argtypes); every entry point of include/ebem.h
PROTOTYPES = {
    "ebem_version": (C.c_int, []),
    "ebem_last_error": (C.c_char_p, []),
    "ebem_release_workspace": (C.c_int, []),
    "ebem_workspace_info": (C.c_int, [C.c_int, C.POINTER(C.c_ulonglong), C.POINTER(C.c_ulonglong)]),
    "ebem_device_release": (C.c_int, [C.c_int]),
    "ebem_profile_enable": (C.c_int, [C.c_int]),
    "ebem_profile_read": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "ebem_mesh_cache_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_longlong)]),
    "ebem_quad_gh": (C.c_int, [C.c_int, C.c_int, C.c_void_p, C.c_void_p]),
    "ebem_mesh_create": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]),
    "ebem_mesh_destroy": (C.c_int, [C.c_void_p]),
    "ebem_mesh_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "ebem_mesh_derived": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "ebem_num_blocks": (C.c_int, [C.c_void_p, C.POINTER(ProblemC), C.POINTER(C.c_int)]),
    "ebem_assemble_sa": (C.c_int, [C.c_void_p, C.POINTER(ProblemC), C.c_int, C.c_int, C.c_int, C.c_void_p,
                                   C.c_int, C.c_void_p, C.POINTER(C.c_longlong)]),
    "ebem_assemble_sa_panel": (C.c_int, [C.c_void_p, C.POINTER(ProblemC), C.c_int, C.c_int, C.c_int, C.c_int,
                                         C.c_int, C.c_void_p, C.c_longlong, C.c_int, C.c_void_p,
                                         C.POINTER(C.c_longlong)]),
    "ebem_assemble_ghc": (C.c_int, [C.c_void_p, C.POINTER(ProblemC), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                    C.c_void_p, C.c_int, C.c_void_p]),
    "ebem_rhs": (C.c_int, [C.c_void_p, C.POINTER(ProblemC), C.c_int, C.c_int, C.c_void_p, C.c_void_p]),
    "ebem_march": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "ebem_march_ex": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p]),
    "ebem_banded_assemble": (C.c_int, [C.c_void_p, C.POINTER(ProblemC), C.c_int, C.c_int, C.c_void_p,
                                       C.POINTER(C.c_void_p)]),
    "ebem_banded_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_longlong),
                                   C.POINTER(C.c_longlong)]),
    "ebem_banded_to_dense": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p]),
    "ebem_banded_march": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "ebem_banded_destroy": (None, [C.c_void_p]),
    "ebem_lu_create": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.POINTER(C.c_void_p)]),
    "ebem_lu_solve": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "ebem_lu_destroy": (None, [C.c_void_p]),
    "ebem_history_gemv": (C.c_int, [C.c_void_p, C.c_int, C.c_longlong, C.c_void_p, C.c_void_p, C.c_void_p]),
    "ebem_timemarch_sa": (C.c_int, [C.c_void_p, C.POINTER(ProblemC), C.c_int, C.c_int, C.c_void_p,
                                    C.POINTER(C.c_int), C.c_void_p]),
    "ebem_pp_sa": (C.c_int, [C.c_void_p, C.POINTER(ProblemC), C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                             C.c_void_p, C.c_void_p]),
    "ebem_assemble_sa_noalloc": (C.c_int, [C.c_void_p, C.POINTER(ProblemC), C.c_int, C.c_int, C.c_int, C.c_void_p,
                                           C.c_int, C.c_void_p, C.POINTER(C.c_longlong)]),
    "ebem_batch_create": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                    C.POINTER(C.c_void_p)]),
    "ebem_batch_assemble": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "ebem_batch_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_float),
                                  C.POINTER(C.c_longlong)]),
    "ebem_batch_destroy": (C.c_int, [C.c_void_p]),
    "ebem_sa_pair_blocks": (C.c_int, [C.c_void_p, C.POINTER(ProblemC), C.c_int, C.c_int, C.c_void_p, C.c_longlong,
                                      C.c_int, C.c_void_p, C.c_void_p]),
    "ebem_selector_init": (C.c_int, [C.c_void_p, C.c_ulonglong]),
    "ebem_selector_features": (C.c_int, [C.c_void_p, C.POINTER(ProblemC), C.c_void_p, C.c_longlong, C.c_void_p,
                                         C.c_void_p]),
    "ebem_selector_sweeps": (C.c_int, [C.c_void_p, C.POINTER(ProblemC), C.c_void_p, C.c_longlong, C.c_void_p,
                                       C.c_void_p]),
    "ebem_selector_labels": (C.c_int, [C.c_void_p, C.c_longlong, C.c_double, C.c_double, C.c_void_p, C.c_void_p,
                                       C.c_void_p]),
    "ebem_selector_grad": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_longlong, C.c_void_p, C.c_void_p,
                                     C.c_void_p]),
    "ebem_selector_train": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_longlong, C.c_int, C.c_int, C.c_float,
                                      C.c_ulonglong, C.c_void_p, C.c_void_p]),
    "ebem_selector_infer": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(ProblemC), C.c_float, C.c_int, C.c_int,
                                      C.c_void_p, C.POINTER(C.c_longlong), C.c_void_p]),
    "ebem_assemble_sa_selected": (C.c_int, [C.c_void_p, C.POINTER(ProblemC), C.POINTER(C.c_int), C.c_int, C.c_void_p,
                                            C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                                            C.POINTER(C.c_longlong)]),
    "ebem_assemble_sa_ex": (C.c_int, [C.c_void_p, C.POINTER(ProblemC)] + [C.c_int] * 5 + [C.c_void_p, C.c_longlong,
                                      C.c_int, C.c_int, C.c_void_p, C.POINTER(C.c_longlong)]),
    "ebem_timemarch_sa_ex": (C.c_int, [C.c_void_p, C.POINTER(ProblemC), C.c_int, C.c_int, C.c_int, C.c_void_p,
                                       C.POINTER(C.c_int), C.c_void_p]),
    "ebem_pp_gpu": (C.c_int, [C.c_void_p, C.POINTER(ProblemC), C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p,
                              C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "ebem_num_blocks_dir": (C.c_int, [C.c_void_p, C.POINTER(ProblemC), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "ebem_assemble_k": (C.c_int, [C.c_void_p, C.POINTER(ProblemC)] + [C.c_int] * 7 + [C.c_void_p, C.c_int, C.c_void_p]),
    "ebem_assemble_v": (C.c_int, [C.c_void_p, C.POINTER(ProblemC)] + [C.c_int] * 6 + [C.c_void_p, C.c_void_p]),
    "ebem_march_dn": (C.c_int, [C.c_void_p, C.POINTER(ProblemC), C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                                C.c_void_p, C.c_void_p, C.c_void_p]),
    "ebem_march_dd": (C.c_int, [C.c_void_p, C.POINTER(ProblemC), C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                                C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "ebem_pp_dir": (C.c_int, [C.c_void_p, C.POINTER(ProblemC), C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                              C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "ebem_pp_dir_matrices": (C.c_int, [C.c_void_p, C.POINTER(ProblemC), C.c_int, C.c_int, C.c_int, C.c_void_p,
                                       C.c_double, C.c_void_p, C.c_void_p]),
}


def library_path() -> str:
    return _build.LIB


def load(build_if_missing: bool = True):
    """Load libebem.so (building it when missing and nvcc is available)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = os.environ.get("EBEM_LIBRARY", _build.LIB)
    if path == _build.LIB and (not os.path.exists(path) or _build._stale()):
        if not build_if_missing:
            raise FileNotFoundError(f"{path} is missing; run elastodynamicebem_b200.build.build()")
        _build.build()
    lib = C.CDLL(path)
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


def check(rc: int) -> None:
    if rc != 0:
        msg = load().ebem_last_error()
        raise EbemError(rc, msg.decode() if msg else "")


def problem_struct(prm) -> ProblemC:
    return ProblemC(float(prm.rho), float(prm.mu), float(prm.lam), float(prm.Tfin), int(prm.nT))
