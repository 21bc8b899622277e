"""ctypes front-end of the CPU oracle (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this module, and only as the checker.  The oracle is a C++ restatement of the
reference's MATLAB semi-analytic path (see sa_oracle.hpp / ebem_oracle.cpp for
the file:line each routine follows).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS = {}
# "f64": the restatement in double precision (the reference's own arithmetic);
# "q": the same formulas in binary128 on the same double inputs (arbiter for
# the exact value of the reference's formulas).
_FILES = {"f64": "liboracle.so", "q": "liboracle_q.so"}

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def build() -> str:
    """Compile the oracle (make in this directory); returns the .so path."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return os.path.join(_HERE, "liboracle.so")


def lib(variant: str = "f64"):
    if variant not in _LIBS:
        path = os.path.join(_HERE, _FILES[variant])
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        mesh_args = [_dp, C.c_int, _ip, C.c_int]
        par = [C.c_double, C.c_double, C.c_double, C.c_double, C.c_int]
        L.or_gh.argtypes = [C.c_int, C.c_int, _dp, _dp]
        L.or_gh.restype = C.c_int
        L.or_mesh_derived.argtypes = mesh_args + [_dp, _dp, _dp, _dp]
        L.or_num_blocks.argtypes = [_dp, C.c_int, C.c_double, C.c_double, C.c_int]
        L.or_num_blocks.restype = C.c_int
        L.or_assemble_sa.argtypes = mesh_args + par + [C.c_int, C.c_int, C.c_int, _dp, C.c_int]
        L.or_assemble_sa.restype = C.c_longlong
        L.or_assemble_sa_pairs.argtypes = mesh_args + par + [C.c_int, C.c_int, _ip, _ip, _ip, _dp, C.c_int]
        L.or_rhs.argtypes = mesh_args + par + [C.c_int, C.c_int, _dp]
        L.or_tn_test.argtypes = [C.c_double] * 7 + [C.c_int] * 3 + [_dp]
        L.or_march.argtypes = [_dp, C.c_int, C.c_int, _dp, C.c_int, _dp]
        L.or_march_exact.argtypes = [_dp, C.c_int, C.c_int, _dp, C.c_int, _dp]
        L.or_pp_sa.argtypes = mesh_args + par + [_dp, _dp, C.c_int, _dp, C.c_int, _dp, C.c_int]
        L.or_assemble_ghc.argtypes = mesh_args + par + [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _dp, C.c_int]
        L.or_pp_gpu.argtypes = mesh_args + par + [_dp, _dp, C.c_int, _dp, C.c_int] + [C.c_int] * 4 + [_dp, C.c_int]
        L.or_count_nonnull.argtypes = mesh_args + par + [C.c_int]
        L.or_count_nonnull.restype = C.c_longlong
        L.or_field_integrals.argtypes = [_dp, C.c_int, _ip, C.c_int, C.c_double, C.c_double, C.c_int, _dp,
                                         C.c_double, _dp]
        L.or_field_integrals.restype = C.c_int
        if variant == "f64":
            mat = [C.c_double, C.c_double, C.c_double, C.c_double]    # rho, mu, lambda, dt
            L.or_p1_coeffs.argtypes = mesh_args + [C.c_int, _dp, _dp]
            L.or_doppio_gauss.argtypes = [C.c_int, _dp, _dp]
            L.or_assemble_k.argtypes = mesh_args + mat + [C.c_int] * 7 + [_dp, C.c_int]
            L.or_k_sing.argtypes = mesh_args + mat + [C.c_int] * 4 + [_dp, C.c_int]
            L.or_v_diag.argtypes = mesh_args + mat + [C.c_int] * 4 + [_dp, C.c_int]
            L.or_pp_dir_g.argtypes = mesh_args + mat + [C.c_int, C.c_int, _dp, C.c_double, C.c_int, _dp]
            L.or_pp_dir_p.argtypes = mesh_args + mat + [C.c_int, C.c_int, _dp, C.c_double, _dp]
        _LIBS[variant] = L
    return _LIBS[variant]


def _m(mesh):
    return (np.ascontiguousarray(mesh.coordinates, np.float64), mesh.number_nodes,
            np.ascontiguousarray(mesh.triangles, np.int32), mesh.numberTriangles)


def _p(prm):
    return (float(prm.rho), float(prm.mu), float(prm.lam), float(prm.dt), int(prm.nT))


def gauss_hammer(n_nodes: int, n_sub: int = 1):
    nodes = np.zeros((n_sub * n_nodes, 3))
    w = np.zeros(n_nodes)
    rc = lib().or_gh(n_nodes, n_sub, nodes, w)
    if rc:
        raise ValueError(f"invalid Gauss-Hammer rule ({n_nodes}, {n_sub})")
    return nodes, w


def num_blocks(mesh, prm) -> int:
    vs = (prm.mu / prm.rho) ** 0.5
    return lib().or_num_blocks(np.ascontiguousarray(mesh.coordinates), mesh.number_nodes, vs, prm.dt, prm.nT)


def assemble_sa(mesh, prm, n_gh: int, lag0: int, nlag: int, nthreads: int = 0, variant: str = "f64"):
    n3 = 3 * mesh.numberTriangles
    E = np.zeros(n3 * n3 * nlag)
    nn = lib(variant).or_assemble_sa(*_m(mesh), *_p(prm), n_gh, lag0, nlag, E, nthreads)
    if nn < 0:
        raise ValueError("oracle assembly failed")
    return E.reshape(nlag, n3, n3).transpose(0, 2, 1), int(nn)   # E[l][row, col]


def assemble_sa_pairs(mesh, prm, n_gh: int, src, fld, lag, nthreads: int = 0, variant: str = "f64"):
    src = np.ascontiguousarray(src, np.int32)
    fld = np.ascontiguousarray(fld, np.int32)
    lag = np.ascontiguousarray(lag, np.int32)
    out = np.zeros(9 * len(src))
    lib(variant).or_assemble_sa_pairs(*_m(mesh), *_p(prm), n_gh, len(src), src, fld, lag, out, nthreads)
    return out.reshape(len(src), 3, 3).transpose(0, 2, 1)    # block[q][r, c]


def rhs(mesh, prm, n_gh: int, datum_id: int, variant: str = "f64"):
    n3 = 3 * mesh.numberTriangles
    b = np.zeros(n3 * prm.nT)
    lib(variant).or_rhs(*_m(mesh), *_p(prm), n_gh, datum_id, b)
    return b.reshape(prm.nT, n3).T.copy()        # (3N, nT)


def tn_test(x1: float, x2: float, t0: float, t1: float, prm, nang: int = 24, nsplit: int = 4, nrad: int = 24):
    """The reference's manufactured 'TEST' boundary value at (x1, x2) for the
    instants (t0, t1) (BEMenerg_core_calcNucleoTn.m:13-132), length 3."""
    out = np.zeros(3)
    if lib().or_tn_test(x1, x2, t0, t1, prm.rho, prm.mu, prm.lam, nang, nsplit, nrad, out):
        raise ValueError("TEST datum: point outside the screen or bad rule")
    return out


def march(E, b):
    """E: (L, 3N, 3N) with E[l][row, col]; b: (3N, nT).  Returns phi (3N, nT)."""
    L, n3, _ = E.shape
    nT = b.shape[1]
    Ecm = np.ascontiguousarray(E.transpose(0, 2, 1)).ravel()
    bcm = np.ascontiguousarray(b.T).ravel()
    phi = np.zeros(n3 * nT)
    rc = lib().or_march(Ecm, n3, L, bcm, nT, phi)
    if rc:
        raise ValueError("singular E_0")
    return phi.reshape(nT, n3).T.copy()


def march_exact(E, b, variant: str = "q"):
    """The marching of `march` with the factorisation, history sums and
    solves in binary128 (variant "q") on the given double data."""
    L, n3, _ = E.shape
    nT = b.shape[1]
    Ecm = np.ascontiguousarray(E.transpose(0, 2, 1)).ravel()
    bcm = np.ascontiguousarray(b.T).ravel()
    phi = np.zeros(n3 * nT)
    if lib(variant).or_march_exact(Ecm, n3, L, bcm, nT, phi):
        raise ValueError("singular E_0")
    return phi.reshape(nT, n3).T.copy()


def pp_sa(mesh, prm, phi, points, times, nthreads: int = 0, variant: str = "f64"):
    """u(x, t): returns (3, npts, ntimes)."""
    n3 = 3 * mesh.numberTriangles
    phicm = np.ascontiguousarray(np.asarray(phi).T).ravel()
    pts = np.ascontiguousarray(points, np.float64)
    tms = np.ascontiguousarray(times, np.float64)
    u = np.zeros(3 * len(pts) * len(tms))
    lib(variant).or_pp_sa(*_m(mesh), *_p(prm), phicm, pts, len(pts), tms, len(tms), u, nthreads)
    return u.reshape(len(tms), len(pts), 3).transpose(2, 1, 0).copy()


def pp_gpu(mesh, prm, phi, points, times, n_sub: int, n_sing: int, variant: int, stride: int | None = None,
           nthreads: int = 0):
    """The reference's numerical post-processing restated (variant 0:
    kernelSP with its host sum, node stride 3 unless given; 1: kernelLayer):
    u (3, npts, ntimes)."""
    if stride is None:
        stride = 3 if variant == 0 else n_sing
    phicm = np.ascontiguousarray(np.asarray(phi).T).ravel()
    pts = np.ascontiguousarray(points, np.float64)
    tms = np.ascontiguousarray(times, np.float64)
    u = np.zeros(3 * len(pts) * len(tms))
    rc = lib().or_pp_gpu(*_m(mesh), *_p(prm), phicm, pts, len(pts), tms, len(tms), n_sub, n_sing, variant, stride, u,
                         nthreads)
    if rc:
        raise ValueError(f"invalid post-processing rule ({rc})")
    return u.reshape(len(tms), len(pts), 3).transpose(2, 1, 0).copy()


def assemble_ghc(mesh, prm, n_gh: int, n_sub: int, n_sing: int, lag0: int, nlag: int, nthreads: int = 0):
    n3 = 3 * mesh.numberTriangles
    E = np.zeros(n3 * n3 * nlag)
    rc = lib().or_assemble_ghc(*_m(mesh), *_p(prm), n_gh, n_sub, n_sing, lag0, nlag, E, nthreads)
    if rc:
        raise ValueError("invalid rule")
    return E.reshape(nlag, n3, n3).transpose(0, 2, 1)


def count_nonnull(mesh, prm, L: int) -> int:
    return int(lib().or_count_nonnull(*_m(mesh), *_p(prm), L))


_CLIB = None


def flop_census(mesh, prm, n_gh: int, npairs: int = 2000, seed: int = 0, L: int | None = None):
    """FP64 operation census of the SA path on a seeded sample of (source,
    field) pairs.  Returns a dict with flops per evaluated (pair, level), per
    non-null pair-lag under level reuse and under the reference's
    three-instants-per-lag schedule, and the transcendental share."""
    global _CLIB
    if _CLIB is None:
        path = os.path.join(_HERE, "liboracle_count.so")
        if not os.path.exists(path):
            build()
        _CLIB = C.CDLL(path)
        _CLIB.or_flop_census.argtypes = [_dp, C.c_int, _ip, C.c_int, _dp, _dp, _dp, _dp,
                                         C.c_double, C.c_double, C.c_double, C.c_int, C.c_int, _dp, _dp,
                                         C.c_int, _ip, _ip, _dp]
    if L is None:
        L = num_blocks(mesh, prm)
    rng = np.random.default_rng(seed)
    N = mesh.numberTriangles
    src = rng.integers(0, N, npairs).astype(np.int32)
    fld = rng.integers(0, N, npairs).astype(np.int32)
    nodes, w = gauss_hammer(n_gh, 1)
    out = np.zeros(5)
    _CLIB.or_flop_census(*_m(mesh), np.ascontiguousarray(mesh.normal), np.ascontiguousarray(mesh.area),
                         np.ascontiguousarray(mesh.center), np.ascontiguousarray(mesh.maxL),
                         prm.velP, prm.velS, prm.dt, int(L), int(n_gh), np.ascontiguousarray(nodes.ravel()),
                         np.ascontiguousarray(w), npairs, src, fld, out)
    flops, trans, nlev, nlag, fref = out
    return {
        "flops_per_level_eval": flops / max(nlev, 1),
        "level_evals_per_pair_lag": nlev / max(nlag, 1),
        "flops_per_pair_integral": flops / max(nlag, 1),
        "flops_per_pair_integral_reference_schedule": fref / max(nlag, 1),
        "transcendental_share": trans / max(flops, 1),
        "sample_pairs": npairs, "sample_pair_lags": int(nlag),
    }


def field_integrals(mesh, velP: float, velS: float, j: int, x, t: float, variant: str = "f64"):
    """Closed-form ris1..ris6 (each 3x3, global axes) of field triangle j seen
    from point x at time t, and the case id (0 none, 1 SP_SP, 2 SP_P, 3 P)."""
    L = lib(variant)
    out = np.zeros(54)
    typ = L.or_field_integrals(*_m(mesh), float(velP), float(velS), int(j),
                               np.ascontiguousarray(x, np.float64), float(t), out)
    return out.reshape(6, 3, 3), int(typ)


def ref_kernel_ms(name: str) -> float:
    """Device time (CUDA events) of the last launch of the reference kernel
    built into oracle/_ref/libref_<name>.so (ghc, k, g or p)."""
    L = C.CDLL(os.path.join(_HERE, "_ref", f"libref_{name}.so"))
    L.ref_last_kernel_ms.restype = C.c_float
    return float(L.ref_last_kernel_ms())


def ref_ghc_available() -> bool:
    return os.path.exists(os.path.join(_HERE, "_ref", "libref_ghc.so"))


def ref_ghc(mesh, prm, n_gh: int, n_sub: int, n_sing: int, nlag: int):
    """Run the reference's own CUDA kernelGHC (compiled from its source into
    oracle/_ref by `make ref`) on the device: E (nlag, 3N, 3N) with
    E[l][row, col], off-diagonal blocks only, as BEMenerg_coreGPU_launchKernel
    produces them."""
    L = C.CDLL(os.path.join(_HERE, "_ref", "libref_ghc.so"))
    L.ref_ghc.argtypes = [_dp, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, _dp, _dp,
                          C.c_int, _dp, _dp, C.c_int, C.c_int, _dp, _dp, C.c_int, C.c_int]
    N = mesh.numberTriangles
    gn, gw = gauss_hammer(n_gh, 1)
    cn, cw = gauss_hammer(n_sing, n_sub)
    P = mesh.coordinates[mesh.triangles]                  # (N, vertex, coord)
    verts = np.ascontiguousarray(P.transpose(0, 2, 1).reshape(N, 9))   # 9t + 3*coord + vertex
    E = np.zeros(9 * N * N * nlag)
    rc = L.ref_ghc(E, N, nlag, prm.dt, prm.velP, prm.velS, 4 * np.pi * prm.rho, np.ascontiguousarray(gw),
                   np.ascontiguousarray(gn), n_gh, np.ascontiguousarray(cw), np.ascontiguousarray(cn), n_sub, n_sing,
                   verts.ravel(), np.ascontiguousarray(mesh.area), 0, nlag)
    if rc:
        raise RuntimeError(f"reference kernelGHC launch failed ({rc})")
    n3 = 3 * N
    return E.reshape(nlag, n3, n3).transpose(0, 2, 1)


def ref_pp_available() -> bool:
    return all(os.path.exists(os.path.join(_HERE, "_ref", f)) for f in ("libref_sp.so", "libref_layer.so"))


def _pp_inputs(mesh, prm, t, n_sub, n_sing):
    N = mesh.numberTriangles
    nhat = int(np.ceil(t / prm.dt)) - 1
    diff = t - np.arange(nhat + 1) * prm.dt                       # diffTemp of calcSP.m:35 / calcLayer.m:33
    nodes, w = gauss_hammer(n_sing, n_sub)
    P = mesh.coordinates[mesh.triangles]
    verts = np.ascontiguousarray(P.transpose(0, 2, 1).reshape(N, 9)).ravel()
    return (N, nhat, np.ascontiguousarray(diff), np.ascontiguousarray(w), np.ascontiguousarray(nodes), verts,
            np.ascontiguousarray(mesh.area), np.ascontiguousarray(mesh.center).ravel(),
            np.ascontiguousarray(mesh.maxL))


def ref_pp_sp(mesh, prm, phi, x, t: float, n_sub: int, n_sing: int):
    """The reference's kernelSP (compiled from its source into oracle/_ref) for
    one point x and time t, with the host sum of
    BEMenerg_postProcGPU_calcSP.m:78-85 done here: (u (3,), kernel ms)."""
    if t <= 0:
        return np.zeros(3), 0.0
    L = C.CDLL(os.path.join(_HERE, "_ref", "libref_sp.so"))
    L.ref_sp.argtypes = [_dp, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, _dp, _dp, _dp, _dp, C.c_int,
                         C.c_int, _dp, _dp, _dp, _dp]
    L.ref_last_kernel_ms.restype = C.c_float
    N, nhat, diff, w, nodes, verts, area, ctr, maxl = _pp_inputs(mesh, prm, t, n_sub, n_sing)
    numIst = nhat + 1
    M = np.zeros(9 * numIst * N)
    rc = L.ref_sp(M, N, numIst, prm.velP, prm.velS, 4 * np.pi * prm.rho, np.ascontiguousarray(x, np.float64), diff,
                  w, nodes.ravel(), n_sub, n_sing, verts, area, ctr, maxl)
    if rc:
        raise RuntimeError(f"reference kernelSP launch failed ({rc})")
    M = M.reshape(3 * N, 3 * numIst).T                             # [3 numIst x 3N]
    u = np.zeros(3)
    for k in range(nhat):
        u += (M[3 * k:3 * k + 3] - M[3 * k + 3:3 * k + 6]) @ phi[:, k]
    u += M[3 * nhat:3 * nhat + 3] @ phi[:, nhat]
    return u, float(L.ref_last_kernel_ms())


def ref_pp_layer(mesh, prm, phi, pts, t: float, n_sub: int, n_sing: int):
    """The reference's kernelLayer (compiled from its source into oracle/_ref)
    for all points at one time t: (u (3, npts), kernel ms)."""
    pts = np.ascontiguousarray(pts, np.float64)
    if t <= 0:
        return np.zeros((3, len(pts))), 0.0
    L = C.CDLL(os.path.join(_HERE, "_ref", "libref_layer.so"))
    L.ref_layer.argtypes = [_dp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, _dp, _dp, _dp, _dp,
                            C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp]
    L.ref_last_kernel_ms.restype = C.c_float
    N, nhat, diff, w, nodes, verts, area, ctr, maxl = _pp_inputs(mesh, prm, t, n_sub, n_sing)
    numIst = nhat + 1
    dens = np.ascontiguousarray(np.asarray(phi)[:, :numIst]).ravel()   # reshape(density(:,1:numIst)', ...)
    u = np.zeros(3 * len(pts))
    rc = L.ref_layer(u, N, len(pts), numIst, prm.velP, prm.velS, 4 * np.pi * prm.rho, pts.ravel(), diff, w,
                     nodes.ravel(), n_sub, n_sing, verts, area, ctr, maxl, dens)
    if rc:
        raise RuntimeError(f"reference kernelLayer launch failed ({rc})")
    return u.reshape(len(pts), 3).T.copy(), float(L.ref_last_kernel_ms())


def ref_ghc_composite(mesh, prm, n_gh: int, n_sub: int, n_sing: int, nlag: int, max_threads: int = 256):
    """The reference's kernelGHC with an inner composite rule of any size.

    The kernel runs one thread per inner node in a block of (n_sub, n_sing)
    threads with 72 bytes of shared memory each, so a launch holds a few
    hundred nodes at most (registers and the 48 KB shared-memory default).  The
    composite rule is a sum over its sub-triangles, so a larger rule is run as
    consecutive launches over chunks of its sub-triangles (nodes sub * n_sing
    + sing, GaussHammerComposite.m's order) with the full rule's weights; the
    launcher accumulates into the same matrix (E += block, kernelGHC.cu:165).
    Chunks hold a power of two of sub-triangles, as the kernel's shared-memory
    tree reduction over x requires."""
    L = C.CDLL(os.path.join(_HERE, "_ref", "libref_ghc.so"))
    L.ref_ghc.argtypes = [_dp, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, _dp, _dp,
                          C.c_int, _dp, _dp, C.c_int, C.c_int, _dp, _dp, C.c_int, C.c_int]
    N = mesh.numberTriangles
    gn, gw = gauss_hammer(n_gh, 1)
    cn, cw = gauss_hammer(n_sing, n_sub)
    chunk = n_sub
    while chunk * n_sing > max_threads:
        chunk //= 2
    if chunk < 1 or n_sub % chunk:
        raise ValueError("composite rule cannot be split into power-of-two chunks")
    P = mesh.coordinates[mesh.triangles]
    verts = np.ascontiguousarray(P.transpose(0, 2, 1).reshape(N, 9)).ravel()
    E = np.zeros(9 * N * N * nlag)
    for c0 in range(0, n_sub, chunk):
        nodes = np.ascontiguousarray(cn[c0 * n_sing:(c0 + chunk) * n_sing])
        rc = L.ref_ghc(E, N, nlag, prm.dt, prm.velP, prm.velS, 4 * np.pi * prm.rho, np.ascontiguousarray(gw),
                       np.ascontiguousarray(gn), n_gh, np.ascontiguousarray(cw), nodes, chunk, n_sing, verts,
                       np.ascontiguousarray(mesh.area), 0, nlag)
        if rc:
            raise RuntimeError(f"reference kernelGHC launch failed ({rc})")
    n3 = 3 * N
    return E.reshape(nlag, n3, n3).transpose(0, 2, 1)


# ---------------------------------------------------------------------------
# direct formulation (dir_oracle.cpp)

def _mat(prm):
    return (float(prm.rho), float(prm.mu), float(prm.lam), float(prm.dt))


def p1_coeffs(mesh, unit_normal: bool = False):
    """P1 basis of every triangle: phi_k(y) = v[t, k] + M[t, k, :] . y."""
    N = mesh.numberTriangles
    M = np.zeros((N, 3, 3)); v = np.zeros((N, 3))
    lib().or_p1_coeffs(*_m(mesh), int(unit_normal), M.reshape(-1), v.reshape(-1))
    return M, v


def doppio_gauss(n: int):
    nodes = np.zeros((n, 3)); w = np.zeros(n)
    if lib().or_doppio_gauss(n, nodes.reshape(-1), w):
        raise ValueError(f"invalid DIAG rule size {n}")
    return nodes, w


def num_blocks_dir(mesh, prm):
    """(L_V, L_K) of BEMenerg_dir_timeMarchingN.m:10,172."""
    LV = num_blocks(mesh, prm)
    return LV, min(LV + 1, prm.nT)


def assemble_k(mesh, prm, n_gh, n_sub, n_sing, lag0, nlag, nblocks=None, fix=False, nthreads=0):
    """K_l off-singular part (kernelK.cu), returned as K[l][row, col] with
    shape (nlag, 3N, 3Nv)."""
    N, Nv = mesh.numberTriangles, mesh.number_nodes
    if nblocks is None:
        nblocks = num_blocks_dir(mesh, prm)[1]
    K = np.zeros(nlag * 9 * N * Nv)
    rc = lib().or_assemble_k(*_m(mesh), *_mat(prm), n_gh, n_sub, n_sing, lag0, nlag, nblocks, int(fix), K, nthreads)
    if rc:
        raise ValueError("invalid rule")
    return K.reshape(nlag, 3 * Nv, 3 * N).transpose(0, 2, 1)


def k_sing(mesh, prm, n_gh, n_diag, lag0, nlag, nthreads=0):
    """Same-triangle parts of K_l (calcSubBlockSingK.m), shape (nlag, 3N, 3Nv)."""
    N, Nv = mesh.numberTriangles, mesh.number_nodes
    K = np.zeros(nlag * 9 * N * Nv)
    if lib().or_k_sing(*_m(mesh), *_mat(prm), n_gh, n_diag, lag0, nlag, K, nthreads):
        raise ValueError("invalid rule")
    return K.reshape(nlag, 3 * Nv, 3 * N).transpose(0, 2, 1)


def v_diag(mesh, prm, n_gh, n_diag, lag0, nlag, nthreads=0):
    """Diagonal blocks of V_l on the DIAG rule (calcSubBlockDiagV.m), as a
    (nlag, 3N, 3N) array that is zero off the diagonal blocks."""
    N = mesh.numberTriangles
    V = np.zeros(nlag * 9 * N * N)
    if lib().or_v_diag(*_m(mesh), *_mat(prm), n_gh, n_diag, lag0, nlag, V, nthreads):
        raise ValueError("invalid rule")
    return V.reshape(nlag, 3 * N, 3 * N).transpose(0, 2, 1)


def pp_dir_matrices(mesh, prm, n_sub, n_sing, x, t, fix=False):
    """(G, P) of kernelG.cu / kernelP.cu at one point and time: G (3 nHat, 3N),
    P (3 nHat, 3 Nv)."""
    N, Nv = mesh.numberTriangles, mesh.number_nodes
    nhat = int(np.ceil(t / prm.dt)) if t > 0 else 0
    G = np.zeros(9 * nhat * N); Pm = np.zeros(9 * nhat * Nv)
    xs = np.ascontiguousarray(x, np.float64)
    if lib().or_pp_dir_g(*_m(mesh), *_mat(prm), n_sub, n_sing, xs, float(t), int(fix), G):
        raise ValueError("invalid rule for kernelG")
    if lib().or_pp_dir_p(*_m(mesh), *_mat(prm), n_sub, n_sing, xs, float(t), Pm):
        raise ValueError("invalid rule")
    return G.reshape(3 * N, 3 * nhat).T, Pm.reshape(3 * Nv, 3 * nhat).T


def ref_dir_available() -> bool:
    return all(os.path.exists(os.path.join(_HERE, "_ref", f)) for f in ("libref_k.so", "libref_g.so", "libref_p.so"))


def _ref_mesh_arrays(mesh, unit_normal):
    N, Nv = mesh.numberTriangles, mesh.number_nodes
    P = mesh.coordinates[mesh.triangles]
    verts = np.ascontiguousarray(P.transpose(0, 2, 1).reshape(-1))          # 9t + 3*coord + vertex
    normT = np.ascontiguousarray(mesh.normal.reshape(-1))
    ism = np.zeros((Nv, N), np.int32)                                         # s*N + m
    for m_, tri in enumerate(mesh.triangles):
        for k, s in enumerate(tri):
            ism[s, m_] = k + 1
    M, v = p1_coeffs(mesh, unit_normal)
    matc = np.ascontiguousarray(M.transpose(0, 2, 1).reshape(-1))            # 9m + 3j + i = M(i, j)
    return verts, normT, np.ascontiguousarray(ism.reshape(-1)), matc, np.ascontiguousarray(v.reshape(-1))


def ref_k(mesh, prm, n_gh, n_sub, n_sing, nlag, nblocks=None):
    """The reference's own kernelK (compiled into oracle/_ref): (nlag, 3N, 3Nv)."""
    L = C.CDLL(os.path.join(_HERE, "_ref", "libref_k.so"))
    _ip_ = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
    L.ref_k.argtypes = [_dp, C.c_int, C.c_int, C.c_int] + [C.c_double] * 6 + [_dp, _dp, C.c_int, _dp, _dp, C.c_int,
                        C.c_int, _dp, _dp, _dp, _ip_, _dp, _dp, C.c_int, C.c_int, _dp, C.c_double]
    N, Nv = mesh.numberTriangles, mesh.number_nodes
    if nblocks is None:
        nblocks = num_blocks_dir(mesh, prm)[1]
    gn, gw = gauss_hammer(n_gh, 1)
    cn, cw = gauss_hammer(n_sing, n_sub)
    verts, normT, ism, matc, vetc = _ref_mesh_arrays(mesh, False)
    K = np.zeros(9 * N * Nv * nlag)
    rc = L.ref_k(K, N, Nv, nlag, prm.dt, prm.velP, prm.velS, prm.lam, prm.mu, prm.rho, np.ascontiguousarray(gw),
                 np.ascontiguousarray(gn), n_gh, np.ascontiguousarray(cw), np.ascontiguousarray(cn), n_sub, n_sing,
                 verts, np.ascontiguousarray(mesh.area), normT, ism, matc, vetc, 0, nblocks,
                 np.ascontiguousarray(mesh.coordinates.reshape(-1)), float(mesh.maxL.max()))
    if rc:
        raise RuntimeError(f"reference kernelK launch failed ({rc})")
    return K.reshape(nlag, 3 * Nv, 3 * N).transpose(0, 2, 1)


def ref_pp_dir(mesh, prm, n_sub, n_sing, x, t):
    """The reference's own kernelG / kernelP at one (x, t): (G, P)."""
    Lg = C.CDLL(os.path.join(_HERE, "_ref", "libref_g.so"))
    Lp = C.CDLL(os.path.join(_HERE, "_ref", "libref_p.so"))
    _ip_ = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
    Lg.ref_g.argtypes = [_dp, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, _dp, _dp, _dp, _dp, C.c_int,
                         C.c_int, _dp, _dp, _dp, _dp]
    Lp.ref_p.argtypes = [_dp, C.c_int, C.c_int, C.c_int] + [C.c_double] * 6 + [_dp, _dp, _dp, _dp, C.c_int, C.c_int,
                                                                               _dp, _dp, _dp, _ip_, _dp, _dp]
    N, Nv = mesh.numberTriangles, mesh.number_nodes
    nhat = int(np.ceil(t / prm.dt))
    diff = np.ascontiguousarray(t - np.arange(nhat + 2) * prm.dt)
    pn, pw = gauss_hammer(n_sing, n_sub)
    verts, normT, ism, matc, vetc = _ref_mesh_arrays(mesh, True)
    xs = np.ascontiguousarray(x, np.float64)
    G = np.zeros(9 * nhat * N); P = np.zeros(9 * nhat * Nv)
    rc = Lg.ref_g(G, N, nhat, prm.velP, prm.velS, prm.rho, xs, diff, np.ascontiguousarray(pw), np.ascontiguousarray(pn),
                  n_sub, n_sing, verts, np.ascontiguousarray(mesh.area), np.ascontiguousarray(mesh.center.reshape(-1)),
                  np.ascontiguousarray(mesh.maxL))
    if rc:
        raise RuntimeError(f"reference kernelG launch failed ({rc})")
    rc = Lp.ref_p(P, N, Nv, nhat, prm.velP, prm.velS, prm.lam, prm.mu, prm.rho, prm.dt, xs, diff,
                  np.ascontiguousarray(pw), np.ascontiguousarray(pn), n_sub, n_sing, verts,
                  np.ascontiguousarray(mesh.area), normT, ism, matc, vetc)
    if rc:
        raise RuntimeError(f"reference kernelP launch failed ({rc})")
    return G.reshape(3 * N, 3 * nhat).T, P.reshape(3 * Nv, 3 * nhat).T
