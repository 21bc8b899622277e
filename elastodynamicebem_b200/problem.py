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
DATUM_TEST = 8              # manufactured: solution phi = (1, 1, 1) on [-1,1]^2 ('TEST')


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


def graded_workload(nx: int = 32, ny: int = 64) -> Workload:
    """Screen [-0.5,0.5]^2 graded toward the edges with exponent 2 (nx x ny
    squares, 2 nx ny triangles: 4096 by default), rho=1, mu=1, lambda=2,
    dt=0.0125, T=1 (80 steps), 7-point outer rule, g=(0,0,t^4 e^-2t);
    displacement at 100 seeded points on z=0.3 at t_n, n=1..80."""
    m = _mesh.screen_graded(nx, ny, 2.0)
    prm = ProblemParams(1.0, 1.0, 2.0, 1.0, 80)
    rng = np.random.default_rng(1)
    pts = np.column_stack([rng.uniform(-0.5, 0.5, 100), rng.uniform(-0.5, 0.5, 100), np.full(100, 0.3)])
    times = prm.dt * np.arange(1, prm.nT + 1)
    return Workload(f"graded_n{m.numberTriangles}", m, prm, 7, DATUM_SCREEN_T4EXP, pts, times)


# ---------------------------------------------------------------------------
# direct formulation: the 1-D bar data of the reference and the bar workload

def _bar_terms(prm: ProblemParams, h: float):
    khat = int(np.ceil(prm.velP * prm.Tfin / (2 * h))) - 1
    return np.arange(0, khat + 1)


def bar_neumann(mesh: _mesh.Mesh, prm: ProblemParams, h: float) -> np.ndarray:
    """Neumann datum gV (nT, 3N) of the bar of height h at the triangle
    centres, t_n = n dt, n = 1..nT (BEMenerg_dir_calcBoundDataNeumann.m:6-24):
    g = (0, 0, 2 mu P(x, t) n_3), P = sum_k (-1)^k [H(c_P t - 2hk - (h - x_3))
    + H(c_P t - 2h(k+1) + (h - x_3))]."""
    k = _bar_terms(prm, h)
    sgn = (-1.0) ** k
    x3 = mesh.center[:, 2]
    out = np.zeros((prm.nT, 3 * mesh.numberTriangles))
    for n in range(1, prm.nT + 1):
        ct = prm.velP * (n * prm.dt)
        a = ((ct - 2 * h * k[None, :] - (h - x3[:, None])) > 0).astype(float)
        b = ((ct - 2 * h * (k[None, :] + 1) + (h - x3[:, None])) > 0).astype(float)
        P = (sgn[None, :] * (a + b)).sum(1)
        out[n - 1, 2::3] = 2 * prm.mu * P * mesh.normal[:, 2]
    return out


def bar_dirichlet(mesh: _mesh.Mesh, prm: ProblemParams, h: float) -> np.ndarray:
    """Dirichlet datum gK (nT, 3Nv) of the bar at the vertices
    (BEMenerg_dir_calcBoundDataDirichlet.m:6-16): g = (0, 0, u(x, t)),
    u = sum_k (-1)^k [(c_P t - 2hk - (h - x_3))_+ - (c_P t - 2h(k+1) + (h - x_3))_+]."""
    k = _bar_terms(prm, h)
    sgn = (-1.0) ** k
    x3 = mesh.coordinates[:, 2]
    out = np.zeros((prm.nT, 3 * mesh.number_nodes))
    for n in range(1, prm.nT + 1):
        ct = prm.velP * (n * prm.dt)
        a = ct - 2 * h * k[None, :] - (h - x3[:, None])
        b = ct - 2 * h * (k[None, :] + 1) + (h - x3[:, None])
        u = (sgn[None, :] * (a * (a > 0) - b * (b > 0))).sum(1)
        out[n - 1, 2::3] = u
    return out


def bar_workload(h: float = 0.1) -> Workload:
    """Prism [0,1] x [0,1] x [0,3] triangulated with squares of side h (h=0.1:
    2800 triangles, 1402 vertices), rho=1, mu=1, lambda=2, dt=0.02, T=2 (100
    steps); Neumann datum of the bar of height 3 (DN formulation);
    displacement at 512 interior points (uniform in the open prism, seed 3) at
    t_n = n dt."""
    m = _mesh.prism_bar(1.0, 1.0, 3.0, h)
    prm = ProblemParams(1.0, 1.0, 2.0, 2.0, 100)
    rng = np.random.default_rng(3)
    pts = np.column_stack([rng.uniform(0, 1, 512), rng.uniform(0, 1, 512), rng.uniform(0, 3, 512)])
    times = prm.dt * np.arange(1, prm.nT + 1)
    return Workload(f"bar_n{m.numberTriangles}", m, prm, 7, DATUM_BAR_H3, pts, times)


# ---------------------------------------------------------------------------
# batched instances

def batch_workload(count: int = 64, seed: int = 4, n_min: int = 128, n_max: int = 2048):
    """Independent screen / sphere instances of uneven size: type alternating
    (screen, sphere), N log-uniform in [n_min, n_max] rounded to the nearest
    generator size (screen 2 n^2, icosphere 20 4^k), dt uniform in
    [0.02, 0.08] rounded to nT = round(1/dt) steps of T = 1, rho = mu = 1,
    lambda = mu U[0.5, 3].  Returns a list of (name, mesh, params)."""
    rng = np.random.default_rng(seed)
    spheres = [k for k in range(0, 6) if n_min <= 20 * 4 ** k <= n_max]
    out = []
    for c in range(count):
        target = math.exp(rng.uniform(math.log(n_min), math.log(n_max)))
        nT = max(1, int(round(1.0 / rng.uniform(0.02, 0.08))))
        lam = float(rng.uniform(0.5, 3.0))
        if c % 2 == 0 or not spheres:
            n = max(2, int(round(math.sqrt(target / 2))))
            m = _mesh.screen_uniform(n)
            name = f"screen_n{m.numberTriangles}"
        else:
            k = min(spheres, key=lambda k: abs(math.log(20 * 4 ** k / target)))
            m = _mesh.icosphere(k)
            name = f"sphere_n{m.numberTriangles}"
        out.append((name, m, ProblemParams(1.0, 1.0, lam, 1.0, nT)))
    return out
