"""Generate the golden fixtures at the benchmark configurations (test data).

Like make_golden.py, the exact value is the oracle restatement of the
reference's formulas evaluated in binary128 ("q") on the same double inputs;
the FP64 restatement's values are stored beside it for the record.

    python tests/golden/make_golden_bench.py   # writes tests/golden/bench_configs.npz

Contents:
  screen128/phi_exact   time-marched density of the screen benchmark (128
                        triangles, rho=1 mu=1 lambda=2, dt=0.05, 20 steps,
                        GH7, datum g=(0,0,t^4 e^-2t)): all 20 blocks E_0..E_19
                        assembled in binary128, right-hand side, then the LU
                        marching carried out in binary128 (3N x nT)
  screen128/u_exact     displacement at the workload's 100 seeded points on
                        z=0.3 at t_n, n=1..20, closed-form post-processing in
                        binary128 of phi_exact (3 x 100 x 20)
  screen128/phi_f64, u_f64   the same chain in the FP64 restatement
  sphere1280_gh{7,12}/{src,fld,lag,exact,f64}
                        300 seeded non-null (source, field, lag) blocks of the
                        headline sphere (icosphere 3, 1280 triangles, lambda=1,
                        dt=0.025, 40 steps), a fifth of them diagonal
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, HERE)

OUT = os.path.join(HERE, "bench_configs.npz")


def screen_chain(variant: str):
    import oracle as O
    from elastodynamicebem_b200 import problem
    w = problem.screen_workload()
    m, prm = w.mesh, w.params
    L = O.num_blocks(m, prm)
    E, _ = O.assemble_sa(m, prm, w.n_gh, 0, L, variant=variant)
    b = O.rhs(m, prm, w.n_gh, w.datum, variant=variant)
    phi = O.march_exact(E, b, variant) if variant == "q" else O.march(E, b)
    u = O.pp_sa(m, prm, phi, w.points, w.times, variant=variant)
    return phi, u


def sphere_sample(n_gh: int, seed: int, q: int = 300):
    import oracle as O
    import make_golden
    from elastodynamicebem_b200 import problem
    w = problem.sphere_workload(n_gh)
    m, prm = w.mesh, w.params
    L = O.num_blocks(m, prm)
    src, fld, lag = make_golden.sample(m, prm, L, q, seed)
    exact = O.assemble_sa_pairs(m, prm, n_gh, src, fld, lag, variant="q")
    f64 = O.assemble_sa_pairs(m, prm, n_gh, src, fld, lag, variant="f64")
    return src, fld, lag, exact, f64


def main():
    import oracle as O
    O.build()
    data = {}
    t0 = time.time()
    phi_q, u_q = screen_chain("q")
    phi_f, u_f = screen_chain("f64")
    data["screen128/phi_exact"], data["screen128/u_exact"] = phi_q, u_q
    data["screen128/phi_f64"], data["screen128/u_f64"] = phi_f, u_f
    print(f"screen128: density f64 vs exact {np.linalg.norm(phi_f - phi_q) / np.linalg.norm(phi_q):.2e}, "
          f"displacement {np.linalg.norm(u_f - u_q) / np.linalg.norm(u_q):.2e} ({time.time() - t0:.0f} s)")
    for n_gh, seed in ((7, 1280), (12, 1281)):
        src, fld, lag, exact, f64 = sphere_sample(n_gh, seed)
        key = f"sphere1280_gh{n_gh}"
        data[f"{key}/src"], data[f"{key}/fld"], data[f"{key}/lag"] = src, fld, lag
        data[f"{key}/exact"], data[f"{key}/f64"] = exact, f64
        print(f"{key}: f64 vs exact {np.linalg.norm(f64 - exact) / np.linalg.norm(exact):.2e}")
    np.savez_compressed(OUT, **data)
    print(f"wrote {OUT} ({os.path.getsize(OUT) / 1e3:.0f} kB, {time.time() - t0:.0f} s)")


if __name__ == "__main__":
    main()
