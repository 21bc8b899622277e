"""MATLAB v5 ``.mat`` files in the reference's output layout.

The reference saves its results with MATLAB ``save``:

* the density, ``density`` (3N x nT), to
  ``./outputData/<domainType><lev>_<method>_<nGH>_density.mat``
  (functions/BEMenerg_indir/BEMenerg_core/BEMenerg_coreSA/BEMenerg_coreSA_timeMarching.m:117,
  BEMenerg_coreGPU/BEMenerg_coreGPU_timeMarching.m:173-174);
* a Toeplitz block, ``matrix`` (3N x 3N), to
  ``./tempData/<domainType><lev>_SA_<nGH>_matrixE<l>.mat``
  (BEMenerg_coreSA_timeMarching.m:42-43);
* a post-processed field, ``campoVett``: a cell array [numPoints x numTimes]
  of 3 x 1 displacements, to ``./outputData/<domainType><lev>_<tag>_campoVett.mat``
  (f/BEMenerg_indir/BEMenerg_postProc/BEMenerg_postProcA/BEMenerg_postProcA_setup.m:18-22,
  tag "A"; f/BEMenerg_dirPP/BEMenerg_ppN_setup.m:20-24, tag "NEW").

These writers produce the same variables, so MATLAB code that loads the
reference's files reads this library's results unchanged.  The arrays here
are the library's: the density as returned by ``core.timemarch_sa``
(nT x 3N, one row per step), blocks as E[l][row, col], displacements as
returned by ``core.pp_sa`` (times x points x 3).
"""
from __future__ import annotations

import os

import numpy as np


def _sio():
    import scipy.io
    return scipy.io


def output_stem(domain_type: str, lev: int, method: str, n_gh: int | None = None, root: str = "./outputData") -> str:
    """``<root>/<domainType><lev>_<method>[_<nGH>]`` as built by the reference's
    ``strcat("./outputData/", pbParam.domainType, num2str(pbParam.lev), ...)``."""
    tail = f"_{method}" + (f"_{n_gh}" if n_gh is not None else "")
    return os.path.join(root, f"{domain_type}{lev}{tail}")


def _host(a) -> np.ndarray:
    if hasattr(a, "detach"):
        a = a.detach().cpu().numpy()
    return np.asarray(a, dtype=np.float64)


def save_density(path: str, density) -> None:
    """Write ``density`` (3N x nT) from the library's (nT, 3N) steps."""
    d = _host(density)
    if d.ndim != 2:
        raise ValueError("density must be (nT, 3N)")
    _sio().savemat(path, {"density": np.ascontiguousarray(d.T)}, format="5", do_compression=False)


def load_density(path: str) -> np.ndarray:
    """Read ``density`` (3N x nT) back as (nT, 3N)."""
    return np.ascontiguousarray(_sio().loadmat(path)["density"].T)


def save_matrix_block(path: str, block) -> None:
    """Write one Toeplitz block E_l[row, col] as ``matrix`` (3N x 3N)."""
    b = _host(block)
    if b.ndim != 2 or b.shape[0] != b.shape[1]:
        raise ValueError("block must be square (3N x 3N)")
    _sio().savemat(path, {"matrix": b}, format="5", do_compression=False)


def load_matrix_block(path: str) -> np.ndarray:
    return np.asarray(_sio().loadmat(path)["matrix"])


def save_campo_vett(path: str, u) -> None:
    """Write displacements u[time, point, comp] as ``campoVett``: a
    numPoints x numTimes cell array of 3 x 1 columns."""
    a = _host(u)
    if a.ndim != 3 or a.shape[2] != 3:
        raise ValueError("u must be (numTimes, numPoints, 3)")
    nt, npts, _ = a.shape
    cell = np.empty((npts, nt), dtype=object)
    for p in range(npts):
        for q in range(nt):
            cell[p, q] = a[q, p].reshape(3, 1).copy()
    _sio().savemat(path, {"campoVett": cell}, format="5", do_compression=False)


def load_campo_vett(path: str) -> np.ndarray:
    """Read ``campoVett`` back as u[time, point, comp]."""
    cell = _sio().loadmat(path)["campoVett"]
    npts, nt = cell.shape
    out = np.empty((nt, npts, 3))
    for p in range(npts):
        for q in range(nt):
            out[q, p] = np.asarray(cell[p, q], dtype=np.float64).reshape(3)
    return out
