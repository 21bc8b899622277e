"""Device-side operators over the C ABI.

torch provides device memory and streams here; every compute step is a
libebem kernel reached through ctypes with plain pointers.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import lib as _lib
from .mesh import Mesh
from .problem import ProblemParams


def _stream_ptr(stream) -> int:
    if stream is None:
        stream = torch.cuda.current_stream()
    return int(stream.cuda_stream)


class DeviceMesh:
    """A mesh uploaded to the current CUDA device (an ``ebem_mesh`` handle)."""

    def __init__(self, mesh: Mesh):
        L = _lib.load()
        self.mesh = mesh
        self._h = C.c_void_p()
        coords = np.ascontiguousarray(mesh.coordinates, np.float64)
        tris = np.ascontiguousarray(mesh.triangles, np.int32)
        _lib.check(L.ebem_mesh_create(coords.ctypes.data, mesh.number_nodes, tris.ctypes.data,
                                      mesh.numberTriangles, C.byref(self._h)))

    @property
    def handle(self):
        return self._h

    @property
    def N(self) -> int:
        return self.mesh.numberTriangles

    def derived(self):
        N = self.N
        n = np.zeros((N, 3)); a = np.zeros(N); c = np.zeros((N, 3)); m = np.zeros(N)
        _lib.check(_lib.load().ebem_mesh_derived(self._h, n.ctypes.data, a.ctypes.data, c.ctypes.data, m.ctypes.data))
        return n, a, c, m

    def close(self):
        if self._h:
            _lib.load().ebem_mesh_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def quad_gh(n_nodes: int, n_sub: int = 1):
    nodes = np.zeros((n_sub * n_nodes, 3))
    w = np.zeros(n_nodes)
    _lib.check(_lib.load().ebem_quad_gh(n_nodes, n_sub, nodes.ctypes.data, w.ctypes.data))
    return nodes, w


def num_blocks(dmesh: DeviceMesh, prm: ProblemParams) -> int:
    L = C.c_int()
    p = _lib.problem_struct(prm)
    _lib.check(_lib.load().ebem_num_blocks(dmesh.handle, C.byref(p), C.byref(L)))
    return int(L.value)


PREC_FP64 = 0
PREC_MIXED = 1


def assemble_sa(dmesh: DeviceMesh, prm: ProblemParams, n_gh: int, lag0: int = 0, nlag: int | None = None,
                out: torch.Tensor | None = None, accumulate: bool = False, stream=None, count: bool = False,
                prec: int = PREC_FP64):
    """E_lag0..E_{lag0+nlag-1} on the device.

    Returns a tensor ``E`` of shape (nlag, 3N, 3N) with ``E[l][row, col]``
    (a transposed view of the column-major C-ABI buffer), and the number of
    non-null pair-lags when ``count`` is set.  ``prec`` selects FP64 or the
    FP32-bulk / FP64-inner mixed mode.
    """
    if nlag is None:
        nlag = num_blocks(dmesh, prm) - lag0
    n3 = 3 * dmesh.N
    if out is None:
        out = torch.empty((nlag, n3, n3), dtype=torch.float64, device="cuda")
    if out.dtype != torch.float64 or not out.is_contiguous() or out.numel() != nlag * n3 * n3:
        raise ValueError("out must be a contiguous float64 tensor of nlag*(3N)^2 elements")
    p = _lib.problem_struct(prm)
    cnt = C.c_longlong(0)
    _lib.check(_lib.load().ebem_assemble_sa_ex(dmesh.handle, C.byref(p), int(n_gh), int(lag0), int(nlag), 0,
                                               dmesh.N, out.data_ptr(), n3, int(bool(accumulate)), int(prec),
                                               _stream_ptr(stream) if out.is_cuda else None,
                                               C.byref(cnt) if count else None))
    E = out.view(nlag, n3, n3).transpose(1, 2)
    return (E, int(cnt.value)) if count else E


def assemble_sa_panel(dmesh: DeviceMesh, prm: ProblemParams, n_gh: int, lag0: int, nlag: int, src0: int, nsrc: int,
                      out: torch.Tensor | None = None, accumulate: bool = False, stream=None, count: bool = False):
    """Source-row panel [src0, src0+nsrc) of E_lag0..: a buffer of nlag x 3N x
    3 nsrc doubles (column-major per lag, leading dimension 3 nsrc).  Returns
    ``(out, nonnull)`` when ``count`` is set, else ``out``."""
    n3 = 3 * dmesh.N
    if out is None:
        out = torch.empty((nlag, n3, 3 * nsrc), dtype=torch.float64, device="cuda")
    if out.dtype != torch.float64 or not out.is_contiguous() or out.numel() != nlag * n3 * 3 * nsrc:
        raise ValueError("out must be a contiguous float64 tensor of nlag*3N*3nsrc elements")
    p = _lib.problem_struct(prm)
    cnt = C.c_longlong(0)
    _lib.check(_lib.load().ebem_assemble_sa_panel(dmesh.handle, C.byref(p), int(n_gh), int(lag0), int(nlag),
                                                  int(src0), int(nsrc), out.data_ptr(), 3 * int(nsrc),
                                                  int(bool(accumulate)),
                                                  _stream_ptr(stream) if out.is_cuda else None,
                                                  C.byref(cnt) if count else None))
    return (out, int(cnt.value)) if count else out


def _ptr(a):
    """Data pointer of a torch tensor or a C-contiguous numpy array."""
    if isinstance(a, torch.Tensor):
        if not a.is_contiguous() or a.dtype != torch.float64:
            raise ValueError("expected a contiguous float64 tensor")
        return a.data_ptr()
    a = np.asarray(a)
    if a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"]:
        raise ValueError("expected a C-contiguous float64 array")
    return a.ctypes.data


def rhs(dmesh: DeviceMesh, prm: ProblemParams, n_gh: int, datum: int, out: torch.Tensor | None = None, stream=None):
    """Right-hand side b (nT, 3N): row n is b_n (column n of the C-ABI's
    column-major 3N x nT array)."""
    n3 = 3 * dmesh.N
    if out is None:
        out = torch.empty((prm.nT, n3), dtype=torch.float64, device="cuda")
    p = _lib.problem_struct(prm)
    _lib.check(_lib.load().ebem_rhs(dmesh.handle, C.byref(p), int(n_gh), int(datum), _ptr(out),
                                    _stream_ptr(stream) if out.is_cuda else None))
    return out


FACTOR_LU = 0
FACTOR_CHOLESKY = 1


def march(E: torch.Tensor, b: torch.Tensor, out: torch.Tensor | None = None, stream=None, factor: int = FACTOR_LU):
    """Density phi (nT, 3N) from the blocks E (L, 3N, 3N storage of
    assemble_sa, i.e. E[l] transposed view) and the right-hand side b (nT, 3N);
    E_0 factored by LU (the reference's) or Cholesky of its symmetric part."""
    Eraw = E.transpose(1, 2).contiguous()      # column-major blocks of the C ABI (no copy for assemble_sa's view)
    L, n3 = Eraw.shape[0], Eraw.shape[1]
    nT = b.shape[0]
    if out is None:
        out = torch.empty((nT, n3), dtype=torch.float64, device=b.device)
    _lib.check(_lib.load().ebem_march_ex(_ptr(Eraw), int(n3), int(L), _ptr(b.contiguous()), int(nT), _ptr(out),
                                         int(factor), _stream_ptr(stream) if out.is_cuda else None))
    return out


class BandedOperator:
    """E_0..E_{L-1} of the semi-analytic method in banded storage on the
    device (ebem_banded_*): per (source, field) pair only its band of non-null
    lags, 6 symmetric entries per block."""

    def __init__(self, dmesh: DeviceMesh, prm: ProblemParams, n_gh: int, prec: int = PREC_FP64, stream=None):
        self.dmesh, self.prm = dmesh, prm
        self._h = C.c_void_p()
        p = _lib.problem_struct(prm)
        _lib.check(_lib.load().ebem_banded_assemble(dmesh.handle, C.byref(p), int(n_gh), int(prec),
                                                    _stream_ptr(stream), C.byref(self._h)))

    def info(self) -> dict:
        n, L, nn, by = C.c_int(), C.c_int(), C.c_longlong(), C.c_longlong()
        _lib.check(_lib.load().ebem_banded_info(self._h, C.byref(n), C.byref(L), C.byref(nn), C.byref(by)))
        return {"N": n.value, "L": L.value, "nonnull": nn.value, "bytes": by.value}

    def to_dense(self, lag0: int = 0, nlag: int | None = None, stream=None) -> torch.Tensor:
        """E[l][row, col], as assemble_sa returns it."""
        L = self.info()["L"]
        nlag = L - lag0 if nlag is None else nlag
        n3 = 3 * self.dmesh.N
        out = torch.empty((nlag, n3, n3), dtype=torch.float64, device="cuda")
        _lib.check(_lib.load().ebem_banded_to_dense(self._h, int(lag0), int(nlag), _ptr(out), _stream_ptr(stream)))
        return out.transpose(1, 2)

    def march(self, b: torch.Tensor, out: torch.Tensor | None = None, stream=None) -> torch.Tensor:
        """Density phi (nT, 3N) from the right-hand side b (nT, 3N)."""
        nT, n3 = b.shape
        if out is None:
            out = torch.empty((nT, n3), dtype=torch.float64, device=b.device)
        _lib.check(_lib.load().ebem_banded_march(self._h, _ptr(b.contiguous()), int(nT), _ptr(out),
                                                 _stream_ptr(stream) if out.is_cuda else None))
        return out

    def close(self):
        if self._h:
            _lib.load().ebem_banded_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DeviceLU:
    """LU factors of the device matrix A[row, col] (ebem_lu_create), kept on
    the device; ``solve`` overwrites contiguous device right-hand sides (one
    per row of ``b``) with A^{-1} b."""

    def __init__(self, A: torch.Tensor, stream=None):
        if A.dim() != 2 or A.shape[0] != A.shape[1] or not A.is_cuda:
            raise ValueError("A must be a square device matrix")
        self.n = int(A.shape[0])
        Acm = A.t().contiguous()                    # column-major storage of A
        self._h = C.c_void_p()
        _lib.check(_lib.load().ebem_lu_create(_ptr(Acm), self.n, _stream_ptr(stream), C.byref(self._h)))

    def solve(self, b: torch.Tensor, stream=None) -> torch.Tensor:
        if not b.is_contiguous() or b.numel() % self.n:
            raise ValueError("b must be contiguous with a multiple of n elements")
        _lib.check(_lib.load().ebem_lu_solve(self._h, _ptr(b), b.numel() // self.n, _stream_ptr(stream)))
        return b

    def close(self):
        if self._h:
            _lib.load().ebem_lu_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def history_gemv(A: torch.Tensor, rows: int, x: torch.Tensor, y: torch.Tensor, stream=None) -> torch.Tensor:
    """y -= A x with A the contiguous column-major storage of a rows x K
    matrix (e.g. lags 1..M of a source-row panel), x (K), y (rows)."""
    K = A.numel() // rows
    if A.numel() != rows * K or x.numel() != K or y.numel() != rows:
        raise ValueError("shape mismatch")
    _lib.check(_lib.load().ebem_history_gemv(_ptr(A), int(rows), int(K), _ptr(x), _ptr(y), _stream_ptr(stream)))
    return y


def timemarch_sa(dmesh: DeviceMesh, prm: ProblemParams, n_gh: int, datum: int, out: torch.Tensor | None = None,
                 stream=None, prec: int = PREC_FP64):
    """BEMenerg_coreSA_timeMarching: assembly + right-hand side + marching.
    Returns (phi (nT, 3N), L)."""
    n3 = 3 * dmesh.N
    if out is None:
        out = torch.empty((prm.nT, n3), dtype=torch.float64, device="cuda")
    p = _lib.problem_struct(prm)
    L = C.c_int()
    _lib.check(_lib.load().ebem_timemarch_sa_ex(dmesh.handle, C.byref(p), int(n_gh), int(datum), int(prec), _ptr(out),
                                                C.byref(L), _stream_ptr(stream) if out.is_cuda else None))
    return out, int(L.value)


def pp_sa(dmesh: DeviceMesh, prm: ProblemParams, phi: torch.Tensor, points, times, stream=None):
    """Displacement u (ntimes, npts, 3) at the points and times from the
    density phi (nT, 3N)."""
    pts = torch.as_tensor(np.ascontiguousarray(points, np.float64)).to(phi.device)
    tms = np.ascontiguousarray(times, np.float64)
    u = torch.empty((len(tms), pts.shape[0], 3), dtype=torch.float64, device=phi.device)
    p = _lib.problem_struct(prm)
    _lib.check(_lib.load().ebem_pp_sa(dmesh.handle, C.byref(p), _ptr(phi.contiguous()), _ptr(pts), int(pts.shape[0]),
                                      tms.ctypes.data, len(tms), _ptr(u),
                                      _stream_ptr(stream) if u.is_cuda else None))
    return u


PP_POINT = 0     # kernelSP semantics: u(x, :) of one point over its times
PP_LAYER = 1     # kernelLayer semantics: u(:, t) of many points at one time


def pp_gpu(dmesh: DeviceMesh, prm: ProblemParams, phi: torch.Tensor, points, times, n_sub: int, n_sing: int,
           variant: int = PP_LAYER, fix_defects: bool = False, stream=None):
    """Numerical post-processing (the reference's method "GPU n_sub n_sing"):
    displacement u (ntimes, npts, 3) from the density phi (nT, 3N)."""
    pts = torch.as_tensor(np.ascontiguousarray(points, np.float64)).to(phi.device)
    tms = np.ascontiguousarray(times, np.float64)
    u = torch.empty((len(tms), pts.shape[0], 3), dtype=torch.float64, device=phi.device)
    p = _lib.problem_struct(prm)
    _lib.check(_lib.load().ebem_pp_gpu(dmesh.handle, C.byref(p), int(n_sub), int(n_sing), int(variant),
                                       1 if fix_defects else 0, _ptr(phi.contiguous()), _ptr(pts),
                                       int(pts.shape[0]), tms.ctypes.data, len(tms), _ptr(u),
                                       _stream_ptr(stream) if u.is_cuda else None))
    return u


def assemble_ghc(dmesh: DeviceMesh, prm: ProblemParams, n_gh: int, n_sub: int, n_sing: int, lag0: int = 0,
                 nlag: int | None = None, out: torch.Tensor | None = None, sa_diagonal: bool = True, stream=None):
    """Numerical-inner E_lag0.. (the reference's GPU method): returns E[l][row, col]
    (added into ``out`` when given, else into zeros)."""
    if nlag is None:
        nlag = num_blocks(dmesh, prm) - lag0
    n3 = 3 * dmesh.N
    if out is None:
        out = torch.zeros((nlag, n3, n3), dtype=torch.float64, device="cuda")
    p = _lib.problem_struct(prm)
    _lib.check(_lib.load().ebem_assemble_ghc(dmesh.handle, C.byref(p), int(n_gh), int(n_sub), int(n_sing), int(lag0),
                                             int(nlag), _ptr(out), int(bool(sa_diagonal)),
                                             _stream_ptr(stream) if out.is_cuda else None))
    return out.view(nlag, n3, n3).transpose(1, 2)


# ---------------------------------------------------------------------------
# direct formulation

FIX_REFERENCE_DEFECTS = 1


def num_blocks_dir(dmesh: DeviceMesh, prm: ProblemParams):
    """(L_V, L_K) of the direct formulation."""
    lv, lk = C.c_int(), C.c_int()
    p = _lib.problem_struct(prm)
    _lib.check(_lib.load().ebem_num_blocks_dir(dmesh.handle, C.byref(p), C.byref(lv), C.byref(lk)))
    return int(lv.value), int(lk.value)


def assemble_k(dmesh: DeviceMesh, prm: ProblemParams, n_gh: int, n_sub: int, n_sing: int, n_diag: int,
               lag0: int = 0, nlag: int | None = None, fix: bool = False, out: torch.Tensor | None = None, stream=None):
    """Double-layer blocks K[l][row, col], shape (nlag, 3N, 3Nv) (a transposed
    view of the column-major storage of the C ABI)."""
    if nlag is None:
        nlag = num_blocks_dir(dmesh, prm)[1] - lag0
    N, Nv = dmesh.N, dmesh.mesh.number_nodes
    if out is None:
        out = torch.empty((nlag, 3 * Nv, 3 * N), dtype=torch.float64, device="cuda")
    p = _lib.problem_struct(prm)
    _lib.check(_lib.load().ebem_assemble_k(dmesh.handle, C.byref(p), int(n_gh), int(n_sub), int(n_sing), int(n_diag),
                                           int(lag0), int(nlag), FIX_REFERENCE_DEFECTS if fix else 0, _ptr(out), 0,
                                           _stream_ptr(stream) if out.is_cuda else None))
    return out.transpose(1, 2)


def assemble_v(dmesh: DeviceMesh, prm: ProblemParams, n_gh: int, n_sub: int, n_sing: int, n_diag: int,
               lag0: int = 0, nlag: int | None = None, out: torch.Tensor | None = None, stream=None):
    """Single-layer blocks of the direct formulation V[l][row, col], (nlag, 3N, 3N)."""
    if nlag is None:
        nlag = num_blocks_dir(dmesh, prm)[0] - lag0
    n3 = 3 * dmesh.N
    if out is None:
        out = torch.empty((nlag, n3, n3), dtype=torch.float64, device="cuda")
    p = _lib.problem_struct(prm)
    _lib.check(_lib.load().ebem_assemble_v(dmesh.handle, C.byref(p), int(n_gh), int(n_sub), int(n_sing), int(n_diag),
                                           int(lag0), int(nlag), _ptr(out),
                                           _stream_ptr(stream) if out.is_cuda else None))
    return out.transpose(1, 2)


def _raw(blocks: torch.Tensor) -> torch.Tensor:
    """Column-major per-lag storage of blocks given as [l][row, col]."""
    return blocks.transpose(1, 2).contiguous()


def march_dn(dmesh: DeviceMesh, prm: ProblemParams, V: torch.Tensor, K: torch.Tensor, gV: torch.Tensor, stream=None):
    """DN time marching: displacement u (nT, 3Nv) from V (LV, 3N, 3N), K (LK, 3N, 3Nv)
    and the Neumann datum gV (nT, 3N)."""
    Vr, Kr = _raw(V), _raw(K)
    u = torch.empty((prm.nT, 3 * dmesh.mesh.number_nodes), dtype=torch.float64, device=Vr.device)
    p = _lib.problem_struct(prm)
    _lib.check(_lib.load().ebem_march_dn(dmesh.handle, C.byref(p), _ptr(Vr), int(Vr.shape[0]), _ptr(Kr),
                                         int(Kr.shape[0]), _ptr(gV.contiguous()), _ptr(u), _stream_ptr(stream)))
    return u


def march_dd(dmesh: DeviceMesh, prm: ProblemParams, V: torch.Tensor, K: torch.Tensor, rhs_: torch.Tensor,
             gK: torch.Tensor, stream=None):
    """DD time marching: traction phi (nT, 3N) from V, K, the right-hand side
    (nT, 3N) and the Dirichlet datum gK (nT, 3Nv)."""
    Vr, Kr = _raw(V), _raw(K)
    phi = torch.empty((prm.nT, 3 * dmesh.N), dtype=torch.float64, device=Vr.device)
    p = _lib.problem_struct(prm)
    _lib.check(_lib.load().ebem_march_dd(dmesh.handle, C.byref(p), _ptr(Vr), int(Vr.shape[0]), _ptr(Kr),
                                         int(Kr.shape[0]), _ptr(rhs_.contiguous()), _ptr(gK.contiguous()), _ptr(phi),
                                         _stream_ptr(stream)))
    return phi


def pp_dir(dmesh: DeviceMesh, prm: ProblemParams, n_sub: int, n_sing: int, a: torch.Tensor, b: torch.Tensor, points,
           times, fix: bool = False, stream=None):
    """Direct post-processing u (ntimes, npts, 3) = sum_n G_n a_n - P_n b_n with
    a (nT, 3N) and b (nT, 3Nv)."""
    pts = torch.as_tensor(np.ascontiguousarray(points, np.float64)).to(a.device)
    tms = np.ascontiguousarray(times, np.float64)
    u = torch.empty((len(tms), pts.shape[0], 3), dtype=torch.float64, device=a.device)
    p = _lib.problem_struct(prm)
    _lib.check(_lib.load().ebem_pp_dir(dmesh.handle, C.byref(p), int(n_sub), int(n_sing),
                                       FIX_REFERENCE_DEFECTS if fix else 0, _ptr(a.contiguous()), _ptr(b.contiguous()),
                                       _ptr(pts), int(pts.shape[0]), tms.ctypes.data, len(tms), _ptr(u),
                                       _stream_ptr(stream)))
    return u


def pp_dir_matrices(dmesh: DeviceMesh, prm: ProblemParams, n_sub: int, n_sing: int, x, t: float, fix: bool = False):
    """The reference's per-(x, t) matrices G (3 nHat, 3N) and P (3 nHat, 3Nv), on the host."""
    N, Nv = dmesh.N, dmesh.mesh.number_nodes
    nhat = int(np.ceil(t / prm.dt)) if t > 0 else 0
    G = np.zeros(9 * nhat * N); P = np.zeros(9 * nhat * Nv)
    xs = np.ascontiguousarray(x, np.float64)
    p = _lib.problem_struct(prm)
    _lib.check(_lib.load().ebem_pp_dir_matrices(dmesh.handle, C.byref(p), int(n_sub), int(n_sing),
                                                FIX_REFERENCE_DEFECTS if fix else 0, xs.ctypes.data, float(t),
                                                G.ctypes.data, P.ctypes.data))
    return G.reshape(3 * N, 3 * nhat).T, P.reshape(3 * Nv, 3 * nhat).T


# ---------------------------------------------------------------------------
# batched assembly

class BatchPlan:
    """Many (mesh, problem) instances assembled by one persistent,
    graph-captured launch (``ebem_batch_*``).  ``assemble()`` returns one
    tensor per instance, E_k[l][row, col] with shape (nlag_k, 3N_k, 3N_k)."""

    def __init__(self, dmeshes, params, n_gh: int, nlag=None, prec: int = PREC_FP64):
        L = _lib.load()
        self.dmeshes = list(dmeshes)
        self.params = list(params)
        n = len(self.dmeshes)
        self._probs = (_lib.ProblemC * n)(*[_lib.problem_struct(p) for p in self.params])
        handles = (C.c_void_p * n)(*[d.handle.value for d in self.dmeshes])
        if nlag is None:
            nlag = [num_blocks(d, p) for d, p in zip(self.dmeshes, self.params)]
        self.nlag = [int(x) for x in nlag]
        nl = (C.c_int * n)(*self.nlag)
        self._h = C.c_void_p()
        _lib.check(L.ebem_batch_create(C.cast(handles, C.c_void_p), C.cast(self._probs, C.c_void_p),
                                       C.cast(nl, C.c_void_p), n, int(n_gh), int(prec), C.byref(self._h)))
        self.outputs = None

    def assemble(self, outputs=None, stream=None):
        if outputs is None:
            if self.outputs is None:
                self.outputs = [torch.empty((l, 3 * d.N, 3 * d.N), dtype=torch.float64, device="cuda")
                                for d, l in zip(self.dmeshes, self.nlag)]
            outputs = self.outputs
        ptrs = (C.c_void_p * len(outputs))(*[o.data_ptr() for o in outputs])
        _lib.check(_lib.load().ebem_batch_assemble(self._h, C.cast(ptrs, C.c_void_p), _stream_ptr(stream)))
        return [o.view(l, 3 * d.N, 3 * d.N).transpose(1, 2) for o, d, l in zip(outputs, self.dmeshes, self.nlag)]

    def info(self):
        w, c, ms, pairs = C.c_int(), C.c_int(), C.c_float(), C.c_longlong()
        _lib.check(_lib.load().ebem_batch_info(self._h, C.byref(w), C.byref(c), C.byref(ms), C.byref(pairs)))
        return {"warps_per_block": w.value, "pairs_per_grab": c.value, "tuned_ms": ms.value, "pairs": pairs.value}

    def close(self):
        if self._h:
            _lib.load().ebem_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# learned quadrature selector

# outer rules of the four classes: (Gauss-Hammer nodes, sub-triangles)
SELECTOR_RULES = ((7, 1), (7, 4), (7, 16), (7, 64))
SELECTOR_PARAMS = 5252


def _rules_arg(rules):
    flat = [int(v) for r in rules for v in r]
    return (C.c_int * len(flat))(*flat), len(rules)


def sa_pair_blocks(dmesh: DeviceMesh, prm: ProblemParams, n_gh: int, n_sub: int, pairs: torch.Tensor, nlag: int,
                   stream=None) -> torch.Tensor:
    """Blocks of explicit pairs (int32 (P, 2) device tensor: source, field)
    at lags 0..nlag-1 with rule (n_gh, n_sub): (P, nlag, 6) float64, the
    symmetric entries 11, 12, 13, 22, 23, 33."""
    pairs = pairs.to(device="cuda", dtype=torch.int32).contiguous()
    out = torch.empty((pairs.shape[0], nlag, 6), dtype=torch.float64, device="cuda")
    p = _lib.problem_struct(prm)
    _lib.check(_lib.load().ebem_sa_pair_blocks(dmesh.handle, C.byref(p), int(n_gh), int(n_sub),
                                               C.c_void_p(pairs.data_ptr()), int(pairs.shape[0]), int(nlag),
                                               C.c_void_p(out.data_ptr()), _stream_ptr(stream)))
    return out


def selector_init(seed: int = 0) -> torch.Tensor:
    """He-initialised MLP parameters (device, float32)."""
    p = torch.empty(SELECTOR_PARAMS, dtype=torch.float32, device="cuda")
    _lib.check(_lib.load().ebem_selector_init(C.c_void_p(p.data_ptr()), int(seed)))
    return p


def selector_features(dmesh: DeviceMesh, prm: ProblemParams, samples: torch.Tensor, stream=None) -> torch.Tensor:
    """Features (n, 12) of samples (int32 (n, 3) device tensor: source, field, lag)."""
    samples = samples.to(device="cuda", dtype=torch.int32).contiguous()
    f = torch.empty((samples.shape[0], 12), dtype=torch.float32, device="cuda")
    p = _lib.problem_struct(prm)
    _lib.check(_lib.load().ebem_selector_features(dmesh.handle, C.byref(p), C.c_void_p(samples.data_ptr()),
                                                  int(samples.shape[0]), C.c_void_p(f.data_ptr()),
                                                  _stream_ptr(stream)))
    return f


def selector_sweeps(dmesh: DeviceMesh, prm: ProblemParams, samples: torch.Tensor, stream=None) -> torch.Tensor:
    """uint8 (n,): 1 where a wavefront sweeps the sample's distance window
    (such lags are assembled on the maximal rule, not by the network)."""
    samples = samples.to(device="cuda", dtype=torch.int32).contiguous()
    f = torch.empty(samples.shape[0], dtype=torch.uint8, device="cuda")
    p = _lib.problem_struct(prm)
    _lib.check(_lib.load().ebem_selector_sweeps(dmesh.handle, C.byref(p), C.c_void_p(samples.data_ptr()),
                                                int(samples.shape[0]), C.c_void_p(f.data_ptr()), _stream_ptr(stream)))
    return f


def selector_labels(blocks: torch.Tensor, tol: float, scale: float, scales: torch.Tensor | None = None,
                    stream=None) -> torch.Tensor:
    """Labels of n samples from their blocks at the four rules ((4, n, 6)
    float64 device tensor); threshold tol * scale, times scales[q] (float64
    device tensor) when given."""
    blocks = blocks.contiguous()
    n = blocks.shape[1]
    y = torch.empty(n, dtype=torch.int32, device="cuda")
    sp = None
    if scales is not None:
        scales = scales.to(device="cuda", dtype=torch.float64).contiguous()
        sp = C.c_void_p(scales.data_ptr())
    _lib.check(_lib.load().ebem_selector_labels(C.c_void_p(blocks.data_ptr()), int(n), float(tol), float(scale), sp,
                                                C.c_void_p(y.data_ptr()), _stream_ptr(stream)))
    return y


def selector_grad(params: torch.Tensor, feats: torch.Tensor, labels: torch.Tensor, stream=None):
    """(gradient, loss) of the mean cross-entropy over the samples."""
    g = torch.empty(SELECTOR_PARAMS, dtype=torch.float32, device="cuda")
    loss = torch.empty(1, dtype=torch.float32, device="cuda")
    _lib.check(_lib.load().ebem_selector_grad(C.c_void_p(params.data_ptr()), C.c_void_p(feats.data_ptr()),
                                              C.c_void_p(labels.data_ptr()), int(labels.numel()),
                                              C.c_void_p(g.data_ptr()), C.c_void_p(loss.data_ptr()),
                                              _stream_ptr(stream)))
    return g, float(loss.item())


def selector_train(params: torch.Tensor, feats: torch.Tensor, labels: torch.Tensor, epochs: int = 20,
                   batch: int = 512, lr: float = 3e-3, seed: int = 0, stream=None):
    """Train in place; returns the per-epoch full-set loss."""
    losses = np.zeros(epochs, dtype=np.float32)
    _lib.check(_lib.load().ebem_selector_train(C.c_void_p(params.data_ptr()), C.c_void_p(feats.data_ptr()),
                                               C.c_void_p(labels.data_ptr()), int(labels.numel()), int(epochs),
                                               int(batch), float(lr), int(seed), losses.ctypes.data,
                                               _stream_ptr(stream)))
    return losses


def selector_infer(params: torch.Tensor, dmesh: DeviceMesh, prm: ProblemParams, threshold: float = 0.9,
                   lag0: int = 0, nlag: int | None = None, stream=None):
    """Class bytes (N*N, nlag) of every (pair, lag), row = field * N + source;
    returns (cls, non-null lags per class)."""
    if nlag is None:
        nlag = num_blocks(dmesh, prm) - lag0
    c = torch.empty((dmesh.N * dmesh.N, nlag), dtype=torch.uint8, device="cuda")
    p = _lib.problem_struct(prm)
    counts = (C.c_longlong * 4)()
    _lib.check(_lib.load().ebem_selector_infer(C.c_void_p(params.data_ptr()), dmesh.handle, C.byref(p),
                                               float(threshold), int(lag0), int(nlag), C.c_void_p(c.data_ptr()),
                                               counts, _stream_ptr(stream)))
    return c, [int(v) for v in counts]


def assemble_sa_selected(dmesh: DeviceMesh, prm: ProblemParams, cls: torch.Tensor, rules=SELECTOR_RULES,
                         lag0: int = 0, nlag: int | None = None, out: torch.Tensor | None = None,
                         prec: int = PREC_FP64, stream=None):
    """E[l][row, col] with each (pair, lag) assembled on the rule of its class
    (cls: uint8 (N*N, nlag) device tensor, row = field * N + source); returns
    (E, non-null lags per class)."""
    if nlag is None:
        nlag = num_blocks(dmesh, prm) - lag0
    n3 = 3 * dmesh.N
    if out is None:
        out = torch.empty((nlag, n3, n3), dtype=torch.float64, device="cuda")
    cls = cls.contiguous()
    if cls.dtype != torch.uint8 or cls.numel() != dmesh.N * dmesh.N * nlag:
        raise ValueError("cls must be a uint8 tensor of N*N*nlag entries")
    p = _lib.problem_struct(prm)
    r, nc = _rules_arg(rules)
    counts = (C.c_longlong * nc)()
    _lib.check(_lib.load().ebem_assemble_sa_selected(dmesh.handle, C.byref(p), r, nc, C.c_void_p(cls.data_ptr()),
                                                     int(lag0), int(nlag), C.c_void_p(out.data_ptr()), int(prec),
                                                     _stream_ptr(stream), counts))
    return out.view(nlag, n3, n3).transpose(1, 2), [int(v) for v in counts]


def assemble_sa_rule(dmesh: DeviceMesh, prm: ProblemParams, n_gh: int, n_sub: int, lag0: int = 0,
                     nlag: int | None = None, out: torch.Tensor | None = None, prec: int = PREC_FP64, stream=None):
    """The plain assembly with the composite outer rule (n_gh, n_sub); returns E."""
    if nlag is None:
        nlag = num_blocks(dmesh, prm) - lag0
    cls = torch.zeros((dmesh.N * dmesh.N, nlag), dtype=torch.uint8, device="cuda")
    E, _ = assemble_sa_selected(dmesh, prm, cls, ((n_gh, n_sub),), lag0, nlag, out, prec, stream)
    return E
