"""Problem parameters (the reference's ``pbParam`` struct) and the benchmark
workload definitions.

``ProblemParams`` mirrors what ``readInputFile``
(functions/utility/fileRead/readInputFile.m:12-74) produces: Lamé parameters,
the wave speeds c_P = sqrt((lambda+2 mu)/rho) and c_S = sqrt(mu/rho)
(``:36,40``), final time and number of time steps (dt = Tfin/nT, as in
``BEMenerg_coreSA_timeMarching.m:15``).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import mesh as _mesh

# Dirichlet data g(x, t) understood by the right-hand-side kernel.  Ids 2..7
# are the reference's cases (BEMenerg_core_calcNucleoTn.m:199-237); 0 and 1
# are the data of the screen and sphere workloads.
DATUM_SCREEN_T4EXP = 0      # g = (0, 0, t^4 exp(-2t))
DATUM_RADIAL_SIN = 1        # g = x sin(2 pi t) H(t)
DATUM_SPHERE_REF = 2        # g = (0, 0, t/2)                      ('sphereUniform')
DATUM_SCREEN_REF = 3        # g = (0, 0, s(t) x1^2), s = sin^5 t before pi/2, 1 after
DATUM_BAR_H1 = 4            # 1-D bar closed form, h = 1            ('barH1')
DATUM_BAR_H3 = 5            # 1-D bar closed form, h = 3            ('barH3')
DATUM_SPHERE_WAVE = 6       # incident Gaussian pulse along x       ('sphereWave')
DATUM_INDUSTRIAL = 7        # incident Gaussian pulse along z       ('elementoIndustriale')


@dataclass
class ProblemParams:
    rho: float
    mu: float
    lam: float
    Tfin: float
    nT: int

    @property
    def dt(self) -> float:
        return self.Tfin / self.nT

    @property
    def velP(self) -> float:
        return math.sqrt((self.lam + 2 * self.mu) / self.rho)

    @property
    def velS(self) -> float:
        return math.sqrt(self.mu / self.rho)


@dataclass
class Workload:
    name: str
    mesh: _mesh.Mesh
    params: ProblemParams
    n_gh: int
    datum: int
    points: np.ndarray       # post-processing points (npts, 3)
    times: np.ndarray        # post-processing times


def screen_workload() -> Workload:
    """Flat screen [-0.5,0.5]^2, 8x8 squares (128 triangles), rho=1, mu=1,
    lambda=2, dt=0.05, T=1 (20 steps), 7-point outer rule, g=(0,0,t^4 e^-2t);
    displacement at 100 seeded points on z=0.3 at t_n, n=1..20."""
    m = _mesh.screen_uniform(8)
    prm = ProblemParams(1.0, 1.0, 2.0, 1.0, 20)
    rng = np.random.default_rng(1)
    pts = np.column_stack([rng.uniform(-0.5, 0.5, 100), rng.uniform(-0.5, 0.5, 100), np.full(100, 0.3)])
    times = prm.dt * np.arange(1, 21)
    return Workload("screen_n128", m, prm, 7, DATUM_SCREEN_T4EXP, pts, times)


def sphere_workload(n_gh: int = 7, subdivisions: int = 3) -> Workload:
    """Unit icosphere subdivided 3x (1280 triangles), rho=1, mu=1, lambda=1,
    dt=0.025, T=1 (40 steps), g = x sin(2 pi t) H(t); displacement at 256
    exterior points (direction uniform on S^2, radius U[1.5, 3], seed 2).
    ``subdivisions`` selects a coarser sphere of the same problem."""
    m = _mesh.icosphere(subdivisions)
    prm = ProblemParams(1.0, 1.0, 1.0, 1.0, 40)
    rng = np.random.default_rng(2)
    d = rng.normal(size=(256, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    pts = d * rng.uniform(1.5, 3.0, 256)[:, None]
    times = prm.dt * np.arange(1, 41)
    return Workload(f"sphere_n{m.numberTriangles}", m, prm, n_gh, DATUM_RADIAL_SIN, pts, times)
