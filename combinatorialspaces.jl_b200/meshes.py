"""Host-side mesh generators and seeded inputs for the workloads (numpy).

Mirrors the reference's CombMeshes generators for this path:

* ``triangulated_grid(lx, ly, dx, dy, compress)`` restates src/CombMeshes.jl:79-133 (vertex
  numbering, triangle gluing with ``glue_triangle!`` semantics, edge orientation false and the
  alternating triangle orientation).
* ``icosahedron()`` is the unit icosahedron glued with ``glue_sorted_triangle!``; the reference
  loads it (``Icosphere(1)``) from a downloaded artifact that this environment does not have.
  Its triangle orientation is left unset, so the library runs ``orient!`` on it.

``uniform(seed, n)`` is the project's input generator (splitmix64 -> uniform[-1, 1)).
"""
from dataclasses import dataclass
from typing import Optional

import numpy as np


@dataclass
class HostMesh:
    points: np.ndarray                 # (nv, 3) float64
    ev0: np.ndarray                    # ∂v0 (target) per edge, 0-based int32
    ev1: np.ndarray                    # ∂v1 (source)
    te0: np.ndarray                    # ∂e0, ∂e1, ∂e2 per triangle
    te1: np.ndarray
    te2: np.ndarray
    edge_orientation: np.ndarray       # int8, 1 / 0
    tri_orientation: Optional[np.ndarray]  # int8, or None (unset: orient! runs)

    @property
    def nv(self):
        return self.points.shape[0]

    @property
    def ne(self):
        return len(self.ev0)

    @property
    def nt(self):
        return len(self.te0)


class _Builder:
    """glue_triangle! / get_edge! (src/SimplicialSets.jl:343-351)."""

    def __init__(self):
        self.ev0, self.ev1, self.tri = [], [], []
        self.emap = {}

    def get_edge(self, src, tgt):
        e = self.emap.get((src, tgt))
        if e is None:
            e = len(self.ev0)
            self.ev1.append(src)   # add_edge!(s, src, tgt): ∂v1 = src, ∂v0 = tgt
            self.ev0.append(tgt)
            self.emap[(src, tgt)] = e
        return e

    def glue(self, v0, v1, v2):
        a = self.get_edge(v0, v1)
        b = self.get_edge(v1, v2)
        c = self.get_edge(v0, v2)
        self.tri.append((b, c, a))  # ∂e0 = e(v1,v2), ∂e1 = e(v0,v2), ∂e2 = e(v0,v1)

    def mesh(self, points, tri_orientation):
        tri = np.asarray(self.tri, np.int32).reshape(-1, 3)
        return HostMesh(np.asarray(points, np.float64), np.asarray(self.ev0, np.int32),
                        np.asarray(self.ev1, np.int32), tri[:, 0].copy(), tri[:, 1].copy(),
                        tri[:, 2].copy(), np.zeros(len(self.ev0), np.int8), tri_orientation)


def _range_len(stop, step):
    r = stop / step
    rr = round(r)
    return (int(rr) if abs(r - rr) <= 1e-10 * max(1.0, abs(r)) else int(np.floor(r))) + 1


def triangulated_grid(lx, ly, dx, dy, compress=True):
    """src/CombMeshes.jl:79-133 with Point3d (z = 0)."""
    scale = lx / (lx + dx / 2)
    shift = dx / 2
    nx, ny = _range_len(lx, dx), _range_len(ly, dy)
    pts = np.zeros((nx * ny, 3))
    for yi in range(1, ny + 1):
        for xi in range(1, nx + 1):
            x = (xi - 1) * dx + shift * (1.0 if yi % 2 == 0 else 0.0)
            if compress:
                x *= scale
            pts[(xi - 1) + nx * (yi - 1)] = (x, (yi - 1) * dy, 0.0)
    b = _Builder()
    for y in range(1, ny):
        for x in range(1, nx):
            i = x + nx * (y - 1)  # 1-based
            if y % 2 == 0:
                b.glue(i - 1, i + nx - 1, i + nx)
                b.glue(i - 1, i, i + nx)
            else:
                b.glue(i - 1, i, i + nx - 1)
                b.glue(i, i + nx - 1, i + nx)
    nxtri, nytri = 2 * (nx - 1), ny - 1
    to = np.zeros(nxtri * nytri, np.int8)
    for y in range(1, nytri + 1):
        o = 0 if y % 2 == 0 else 1
        for x in range(1, nxtri + 1, 2):
            i = x + nxtri * (y - 1) - 1
            to[i] = o
            to[i + 1] = 1 - o
    return b.mesh(pts, to)


def icosahedron():
    """Unit icosahedron (12 vertices, 20 faces), glue_sorted_triangle!, orientation unset."""
    p = (1.0 + 5 ** 0.5) / 2.0
    v = np.array([[-1, p, 0], [1, p, 0], [-1, -p, 0], [1, -p, 0], [0, -1, p], [0, 1, p],
                  [0, -1, -p], [0, 1, -p], [p, 0, -1], [p, 0, 1], [-p, 0, -1], [-p, 0, 1]], float)
    v /= np.sqrt(1.0 + p * p)
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
             (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
             (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    b = _Builder()
    for f in faces:
        b.glue(*sorted(f))
    return b.mesh(v, None)


def uniform(seed, n, dtype=np.float64):
    """splitmix64 stream of `seed` mapped to uniform[-1, 1)."""
    with np.errstate(over="ignore"):
        idx = np.arange(1, n + 1, dtype=np.uint64)
        z = np.uint64(seed) + idx * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return ((z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0) * 2.0 - 1.0).astype(dtype)


def refine_binary(m, radius=0.0):
    """refine(::BinarySubdivision) + propagate_points (src/Multigrid.jl:111-183), vectorised;
    a positive radius projects the new vertices onto that sphere.  Orientation is left unset
    (the library runs orient!, as dualize does on a refined mesh)."""
    nv, ne, nt = m.nv, m.ne, m.nt
    ev0 = np.empty(2 * ne + 3 * nt, np.int32)
    ev1 = np.empty_like(ev0)
    mid = nv + np.arange(ne, dtype=np.int64)
    ev0[0:2 * ne:2] = mid
    ev1[0:2 * ne:2] = m.ev0
    ev0[1:2 * ne:2] = mid
    ev1[1:2 * ne:2] = m.ev1
    e0, e1, e2 = (np.asarray(a, np.int64) for a in (m.te0, m.te1, m.te2))
    m0, m1, m2 = e0 + nv, e1 + nv, e2 + nv
    base = 2 * ne + 3 * np.arange(nt, dtype=np.int64)
    ev0[base], ev1[base] = m1, m0          # m0_m1
    ev0[base + 1], ev1[base + 1] = m2, m1  # m1_m2
    ev0[base + 2], ev1[base + 2] = m2, m0  # m0_m2
    te = np.empty((4 * nt, 3), np.int32)
    b = 4 * np.arange(nt, dtype=np.int64)
    te[b] = np.stack([base + 1, base + 2, base], 1)
    te[b + 1] = np.stack([base + 1, 2 * e2 + 1, 2 * e1 + 1], 1)
    te[b + 2] = np.stack([base + 2, 2 * e2, 2 * e0 + 1], 1)
    te[b + 3] = np.stack([base, 2 * e1, 2 * e0], 1)
    p = np.asarray(m.points, np.float64)
    newp = (p[m.ev0] + p[m.ev1]) / 2
    if radius > 0:
        newp = newp / np.linalg.norm(newp, axis=1, keepdims=True) * radius
    return HostMesh(np.concatenate([p, newp]), ev0, ev1, te[:, 0].copy(), te[:, 1].copy(), te[:, 2].copy(),
                    np.zeros(len(ev0), np.int8), None)


def icosphere(k):
    """Icosphere L_k: the unit icosahedron binary-subdivided k times, new vertices on the unit
    sphere (nv = 10·4^k + 2)."""
    m = icosahedron()
    for _ in range(k):
        m = refine_binary(m, 1.0)
    return m
