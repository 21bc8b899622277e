"""Generate the golden fixtures of the semi-analytic path (test data).

The reference (MATLAB) cannot run here and ships no numeric golden vectors,
so the fixtures hold the exact value of the reference's formulas: the oracle
restatement (oracle/sa_oracle.hpp, routine-by-routine with file:line
citations) evaluated in binary128 on the same double inputs.  For each case
a seeded sample of (source, field, lag) blocks is stored together with the
FP64 restatement's values (the reference's own arithmetic) for the record.

    python tests/golden/make_golden.py        # writes tests/golden/sa_blocks.npz

Cases (generated meshes; nothing is read from the reference):
  screen32_gh{3,7,12,19}  uniform screen 4x4 squares, rho=1 mu=1 lambda=2, dt=0.05, 20 steps
  screen128_gh7           the screen benchmark mesh (8x8 squares)
  sphere80_gh{7,12}       icosphere 1, lambda=1, dt=0.025, 40 steps
  prism28_gh7             box 1x1x3, h=1 (source nodes at distance c_S t = 1 from the opposite face)
  graded48_gh7            graded screen 6x4, exponent 2
  limit32_gh7             lambda = -mu (c_P = c_S)
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def cases():
    from elastodynamicebem_b200 import mesh, problem
    P = problem.ProblemParams
    s4 = mesh.screen_uniform(4)
    out = []
    for g in (3, 7, 12, 19):
        out.append((f"screen32_gh{g}", s4, P(1.0, 1.0, 2.0, 1.0, 20), g))
    out.append(("screen128_gh7", mesh.screen_uniform(8), P(1.0, 1.0, 2.0, 1.0, 20), 7))
    ico = mesh.icosphere(1)
    for g in (7, 12):
        out.append((f"sphere80_gh{g}", ico, P(1.0, 1.0, 1.0, 1.0, 40), g))
    out.append(("prism28_gh7", mesh.prism_bar(1.0, 1.0, 3.0, 1.0), P(1.0, 1.0, 2.0, 2.0, 40), 7))
    out.append(("graded48_gh7", mesh.screen_graded(6, 4), P(1.0, 1.0, 2.0, 1.0, 16), 7))
    out.append(("limit32_gh7", s4, P(1.0, 1.0, -1.0, 1.0, 8), 7))
    return out


def sample(m, prm, L, n, seed):
    """Seeded non-null (source, field, lag) triples, a fifth of them diagonal."""
    rng = np.random.default_rng(seed)
    N = m.numberTriangles
    src, fld, lag = [], [], []
    while len(src) < n:
        i = int(rng.integers(0, N))
        j = i if rng.random() < 0.2 else int(rng.integers(0, N))
        l = int(rng.integers(0, L))
        d = np.linalg.norm(m.center[j] - m.center[i])
        if ((l - 1) * prm.velS * prm.dt < d + m.maxL[i] + m.maxL[j]) and \
           ((l + 1) * prm.velP * prm.dt >= d - m.maxL[i] - m.maxL[j]):
            src.append(i); fld.append(j); lag.append(l)
    return np.array(src, np.int32), np.array(fld, np.int32), np.array(lag, np.int32)


def main():
    import oracle as O
    O.build()
    data = {}
    for k, (name, m, prm, g) in enumerate(cases()):
        L = O.num_blocks(m, prm)
        src, fld, lag = sample(m, prm, L, 400, 100 + k)
        q = O.assemble_sa_pairs(m, prm, g, src, fld, lag, variant="q")
        f = O.assemble_sa_pairs(m, prm, g, src, fld, lag)
        data[f"{name}/src"], data[f"{name}/fld"], data[f"{name}/lag"] = src, fld, lag
        data[f"{name}/exact"], data[f"{name}/f64"] = q, f
        err = np.linalg.norm(f - q) / np.linalg.norm(q)
        print(f"{name:16s} L={L:3d}  FP64 restatement vs exact: {err:.2e}")
    np.savez_compressed(os.path.join(HERE, "sa_blocks.npz"), **data)


if __name__ == "__main__":
    main()
