"""Surface meshes: the Medit ``.mesh`` reader/writer and the generators of the
benchmark geometries.

``read_space_mesh`` mirrors the reference's ``readSpaceMesh``
(functions/utility/fileRead/readSpaceMesh.m:1-151) and ``calcParamMesh``
(functions/utility/fileRead/calcParamMesh.m): the same header skipping, the
same forced boundary label (``readSpaceMesh.m:80-81``) and the same derived
fields — normal n = (P1-P3) x (P2-P3) / |.| (``:114-122``), area (``:119``),
centroid (``:128-130``), longest edge (``:133-139``), the surface curl
(``:146-148``) and the global lMin / lMax.  Triangles are stored 0-based here;
the reference is 1-based.

The generators produce the geometries the benchmark workloads are defined on:
uniform and graded flat screens, the geodesic icosphere and the prism bar.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Mesh:
    coordinates: np.ndarray          # (Nv, 3) float64
    triangles: np.ndarray            # (N, 3) int32, 0-based vertex indices
    normal: np.ndarray = field(default=None)
    area: np.ndarray = field(default=None)
    center: np.ndarray = field(default=None)
    maxL: np.ndarray = field(default=None)
    curl: np.ndarray = field(default=None)
    lMin: float = 0.0
    lMax: float = 0.0
    name: str = ""

    def __post_init__(self):
        self.coordinates = np.ascontiguousarray(self.coordinates, dtype=np.float64)
        self.triangles = np.ascontiguousarray(self.triangles, dtype=np.int32)
        if self.coordinates.ndim != 2 or self.coordinates.shape[1] != 3:
            raise ValueError("coordinates must be (Nv, 3)")
        if self.triangles.ndim != 2 or self.triangles.shape[1] != 3:
            raise ValueError("triangles must be (N, 3)")
        if self.triangles.size and (self.triangles.min() < 0 or self.triangles.max() >= len(self.coordinates)):
            raise ValueError("triangle vertex index out of range")
        self._derive()

    @property
    def number_nodes(self) -> int:
        return int(self.coordinates.shape[0])

    @property
    def numberTriangles(self) -> int:
        return int(self.triangles.shape[0])

    def _derive(self):
        P = self.coordinates[self.triangles]            # (N, 3 vertices, 3)
        vg1 = P[:, 0] - P[:, 2]
        vg2 = P[:, 1] - P[:, 2]
        vg3 = P[:, 0] - P[:, 1]
        n = np.empty_like(vg1)
        n[:, 0] = vg1[:, 1] * vg2[:, 2] - vg2[:, 1] * vg1[:, 2]
        n[:, 1] = -vg1[:, 0] * vg2[:, 2] + vg2[:, 0] * vg1[:, 2]
        n[:, 2] = vg1[:, 0] * vg2[:, 1] - vg2[:, 0] * vg1[:, 1]
        self.area = np.sqrt((n[:, 0] ** 2 + n[:, 1] ** 2) + n[:, 2] ** 2) / 2
        if np.any(self.area <= 0):
            raise ValueError("degenerate triangle (zero area) in mesh")
        self.normal = n / (2 * self.area)[:, None]
        self.center = (P[:, 0] + P[:, 1] + P[:, 2]) / 3
        ln = np.stack([np.linalg.norm(vg3, axis=1), np.linalg.norm(vg2, axis=1), np.linalg.norm(vg1, axis=1)], 1)
        self.maxL = ln.max(1)
        a2 = (2 * self.area)[:, None]
        self.curl = np.stack([vg2 / a2, -vg1 / a2, vg3 / a2], 2)   # (N, 3 comps, 3 cols)
        self.lMin = float(ln.min()) if len(ln) else 0.0
        self.lMax = float(ln.max()) if len(ln) else 0.0

    def vertex_triangle_incidence(self) -> np.ndarray:
        """(Nv, N) boolean incidence: vertex s belongs to triangle m."""
        inc = np.zeros((self.number_nodes, self.numberTriangles), dtype=bool)
        for k in range(3):
            inc[self.triangles[:, k], np.arange(self.numberTriangles)] = True
        return inc


def read_space_mesh(path: str) -> Mesh:
    """Read a Medit ``.mesh`` file the way ``readSpaceMesh.m:13-88`` does."""
    with open(path, "r") as f:
        tok = f.read().split()
    iv = tok.index("Vertices")
    nv = int(tok[iv + 1])
    v = np.array(tok[iv + 2: iv + 2 + 4 * nv], dtype=np.float64).reshape(nv, 4)[:, :3]
    it = tok.index("Triangles")
    nt = int(tok[it + 1])
    t = np.array(tok[it + 2: it + 2 + 4 * nt], dtype=np.float64).reshape(nt, 4)[:, :3].astype(np.int64) - 1
    return Mesh(v, t.astype(np.int32), name=os.path.splitext(os.path.basename(path))[0])


def write_space_mesh(mesh: Mesh, path: str) -> None:
    """Write a Medit ``.mesh`` file that ``read_space_mesh`` (and the reference's reader) accept."""
    with open(path, "w") as f:
        f.write(" MeshVersionFormatted\n 2\n Dimension\n 3\n Vertices\n")
        f.write(f" {mesh.number_nodes}\n")
        for p in mesh.coordinates:
            f.write(f" {p[0]:.17g} {p[1]:.17g} {p[2]:.17g} 0\n")
        f.write(f" Triangles\n {mesh.numberTriangles}\n")
        for t in mesh.triangles:
            f.write(f" {t[0] + 1} {t[1] + 1} {t[2] + 1} 0\n")
        f.write(" End\n")


# --------------------------------------------------------------------------
# generators

def _grid_triangles(nx: int, ny: int, vid) -> list:
    tris = []
    for j in range(ny):
        for i in range(nx):
            a, b, c, d = vid(i, j), vid(i + 1, j), vid(i + 1, j + 1), vid(i, j + 1)
            # counter-clockwise seen from +z: normal (P1-P3)x(P2-P3) points to +z
            tris.append((a, b, d))
            tris.append((b, c, d))
    return tris


def screen_from_axes(xs: np.ndarray, ys: np.ndarray, name: str = "screen") -> Mesh:
    nx, ny = len(xs) - 1, len(ys) - 1
    X, Y = np.meshgrid(xs, ys, indexing="xy")
    coords = np.stack([X.ravel(), Y.ravel(), np.zeros(X.size)], 1)
    tris = _grid_triangles(nx, ny, lambda i, j: j * (nx + 1) + i)
    return Mesh(coords, np.array(tris, dtype=np.int32), name=name)


def screen_uniform(n: int, half: float = 0.5) -> Mesh:
    """[-half, half]^2 at z = 0, n x n squares each split in two (2 n^2 triangles)."""
    xs = np.linspace(-half, half, n + 1)
    return screen_from_axes(xs, xs, name=f"screenUniform_n{n}")


def graded_axis(n: int, grading: float = 2.0, half: float = 0.5) -> np.ndarray:
    """n intervals on [-half, half] graded toward both ends with (k/m)^grading,
    m = n/2 (the rule of the reference's mesh/screenGraded/screengraded.geo)."""
    if n % 2:
        raise ValueError("graded axis needs an even number of intervals")
    m = n // 2
    k = np.arange(m + 1) / m
    left = -half + half * k ** grading
    return np.concatenate([left, -left[-2::-1]])


def screen_graded(nx: int, ny: int, grading: float = 2.0) -> Mesh:
    return screen_from_axes(graded_axis(nx, grading), graded_axis(ny, grading), name=f"screenGraded_{nx}x{ny}")


def icosphere(subdivisions: int, radius: float = 1.0) -> Mesh:
    """Geodesic sphere: icosahedron, each subdivision splits a triangle into 4
    and projects the new vertices on the sphere (20 * 4^k triangles)."""
    t = (1.0 + 5 ** 0.5) / 2
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
         (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
         (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    verts = [np.array(p, float) / np.linalg.norm(p) for p in v]
    faces = list(f)
    for _ in range(subdivisions):
        cache = {}

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                p = verts[a] + verts[b]
                verts.append(p / np.linalg.norm(p))
                cache[key] = len(verts) - 1
            return cache[key]
        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    coords = np.array(verts) * radius
    tris = np.array(faces, dtype=np.int64)
    P = coords[tris]
    n = np.cross(P[:, 0] - P[:, 2], P[:, 1] - P[:, 2])
    flip = (n * P.mean(1)).sum(1) < 0
    tris[flip] = tris[flip][:, [0, 2, 1]]
    return Mesh(coords, tris.astype(np.int32), name=f"icosphere_{subdivisions}")


def prism_bar(lx: float = 1.0, ly: float = 1.0, lz: float = 3.0, h: float = 0.1) -> Mesh:
    """Surface of the box [0,lx] x [0,ly] x [0,lz], structured squares of side
    h split in two, outward normals.  lx=ly=1, lz=3, h=0.1 gives 2800
    triangles and 1402 vertices."""
    nx, ny, nz = int(round(lx / h)), int(round(ly / h)), int(round(lz / h))
    index = {}
    coords = []

    def vid(p):
        key = tuple(int(round(c / h * 1000)) for c in p)
        if key not in index:
            index[key] = len(coords)
            coords.append(p)
        return index[key]
    tris = []

    def face(origin, du, dv, nu, nv, outward):
        o, du, dv = np.array(origin, float), np.array(du, float), np.array(dv, float)
        ids = [[vid(tuple(o + i * du + j * dv)) for j in range(nv + 1)] for i in range(nu + 1)]
        flip = np.dot(np.cross(du, dv), outward) < 0
        for j in range(nv):
            for i in range(nu):
                a, b, c, d = ids[i][j], ids[i + 1][j], ids[i + 1][j + 1], ids[i][j + 1]
                t1, t2 = (a, b, d), (b, c, d)
                if flip:
                    t1, t2 = (a, d, b), (b, d, c)
                tris.extend([t1, t2])
    face((0, 0, 0), (h, 0, 0), (0, h, 0), nx, ny, (0, 0, -1))
    face((0, 0, lz), (h, 0, 0), (0, h, 0), nx, ny, (0, 0, 1))
    face((0, 0, 0), (h, 0, 0), (0, 0, h), nx, nz, (0, -1, 0))
    face((0, ly, 0), (h, 0, 0), (0, 0, h), nx, nz, (0, 1, 0))
    face((0, 0, 0), (0, h, 0), (0, 0, h), ny, nz, (-1, 0, 0))
    face((lx, 0, 0), (0, h, 0), (0, 0, h), ny, nz, (1, 0, 0))
    tris = np.array(tris, dtype=np.int64)
    coords = np.array(coords, float)
    # triangles are consistently outward by construction; (P1-P3)x(P2-P3) must agree
    P = coords[tris]
    n = np.cross(P[:, 0] - P[:, 2], P[:, 1] - P[:, 2])
    ctr = np.array([lx / 2, ly / 2, lz / 2])
    flip = (n * (P.mean(1) - ctr)).sum(1) < 0
    tris[flip] = tris[flip][:, [0, 2, 1]]
    return Mesh(coords, tris.astype(np.int32), name=f"prism_{lx}x{ly}x{lz}_h{h}")
