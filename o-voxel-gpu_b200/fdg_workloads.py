"""Seeded synthetic meshes for the mesh -> flexible-dual-grid workloads.

The reference measures on ``notebooks/test.glb`` (a 268k-vertex / 280k-face
asset that is not distributed with it) and on a subdivided version of it.
These generators build stand-ins with the same sizes and the same kinds of
trouble (open boundaries, overlaps, non-manifold intersections, slivers,
T-junctions).  Every generator is a pure function of its seed.

Conventions (as in the reference example ``examples/mesh2ovox.py``): fp32
vertices, int64 faces, aabb ``[[-0.5]*3, [0.5]*3]`` unless a config says
otherwise, weights ``face_weight=1.0, boundary_weight=0.2,
regularization_weight=1e-2``.

Workloads:
  * ``ico_cap``       -- icosphere level 4 (2562 V / 5120 F), r=0.4, jitter
                         N(0,1e-3), faces inside a random 20 degree cap removed; grid 64.
  * ``primitives``    -- 48 primitives (tori, open cylinders, open boxes,
                         icospheres), scale U(0.05,0.3), random pose inside the
                         aabb, UV-chart seams, 1% sliver faces; ~280k faces; grid 512.
  * ``subdivided``    -- ``primitives`` midpoint-subdivided twice, then a
                         seeded subset subdivided once more (T-junctions), ~10.3M faces.
  * ``sheets``        -- precision stress: near-coplanar stacked sheets,
                         creases of 1..179 degrees, 20% slivers; 200k faces; grid 1024.
  * ``batch``         -- many ``primitives``-style meshes, log-uniform face
                         counts, per-mesh grid and aabb.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

UNIT_AABB = [[-0.5, -0.5, -0.5], [0.5, 0.5, 0.5]]


@dataclass
class Workload:
    name: str
    vertices: np.ndarray  # [V,3] float32
    faces: np.ndarray  # [F,3] int64
    grid_size: int
    aabb: list
    face_weight: float = 1.0
    boundary_weight: float = 0.2
    regularization_weight: float = 1e-2
    meta: dict = field(default_factory=dict)

    @property
    def num_faces(self) -> int:
        return int(self.faces.shape[0])

    def kwargs(self):
        return dict(grid_size=self.grid_size, aabb=self.aabb, face_weight=self.face_weight,
                    boundary_weight=self.boundary_weight, regularization_weight=self.regularization_weight)


# --------------------------------------------------------------------------- primitives
def icosphere(level: int):
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], dtype=np.float64)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
                  [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5],
                  [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], dtype=np.int64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    for _ in range(level):
        v, f = _subdivide_all(v, f)
        v /= np.linalg.norm(v, axis=1, keepdims=True)
    return v, f


def _subdivide_all(v, f):
    """1->4 midpoint subdivision with shared edge midpoints."""
    e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]], axis=0)
    e.sort(axis=1)
    key = e[:, 0] * (v.shape[0] + 1) + e[:, 1]
    uk, inv = np.unique(key, return_inverse=True)
    a = uk // (v.shape[0] + 1)
    b = uk % (v.shape[0] + 1)
    mids = 0.5 * (v[a] + v[b])
    m = (inv + v.shape[0]).reshape(3, -1).T  # m01, m12, m20
    nv = np.concatenate([v, mids], axis=0)
    f0, f1, f2 = f[:, 0], f[:, 1], f[:, 2]
    m01, m12, m20 = m[:, 0], m[:, 1], m[:, 2]
    nf = np.stack([np.stack([f0, m01, m20], 1), np.stack([m01, f1, m12], 1), np.stack([m20, m12, f2], 1),
                   np.stack([m01, m12, m20], 1)], axis=1).reshape(-1, 3)
    return nv, nf


def _grid_mesh(pos_fn, nu, nv, periodic_u, periodic_v, chart):
    """Quad grid over (u,v) parameters, two triangles per quad.  Vertices are
    shared inside a chart of ``chart x chart`` quads and duplicated across chart
    borders (UV seams), as exported assets do."""
    i, j = np.meshgrid(np.arange(nu), np.arange(nv), indexing="ij")
    i = i.ravel()
    j = j.ravel()
    ci, cj = i // chart, j // chart
    ncj = (nv + chart - 1) // chart
    cid = ci * ncj + cj
    side = chart + 1
    corners = []
    for di, dj in ((0, 0), (1, 0), (1, 1), (0, 1)):
        li = i + di - ci * chart
        lj = j + dj - cj * chart
        corners.append(cid * side * side + li * side + lj)
    c = np.stack(corners, 1)
    tri = np.concatenate([c[:, [0, 1, 2]], c[:, [0, 2, 3]]], axis=0)
    ids, inv = np.unique(tri.ravel(), return_inverse=True)
    tri = inv.reshape(-1, 3)
    # parameter coordinates of every unique vertex id
    cid_v = ids // (side * side)
    rem = ids % (side * side)
    li, lj = rem // side, rem % side
    gi = (cid_v // ncj) * chart + li
    gj = (cid_v % ncj) * chart + lj
    u = gi / nu if periodic_u else gi / max(nu, 1)
    w = gj / nv if periodic_v else gj / max(nv, 1)
    return pos_fn(u, w), tri


def torus(rng, n_faces, chart):
    k = int(round(math.sqrt(n_faces / 2.0)))
    R, r = 1.0, rng.uniform(0.2, 0.45)

    def pos(u, w):
        a, b = 2 * np.pi * u, 2 * np.pi * w
        return np.stack([(R + r * np.cos(b)) * np.cos(a), (R + r * np.cos(b)) * np.sin(a), r * np.sin(b)], 1) / (R + r)

    return _grid_mesh(pos, k, k, True, True, chart)


def open_cylinder(rng, n_faces, chart):
    nu = int(round(math.sqrt(n_faces)))
    nvq = max(1, int(round(n_faces / (2 * nu))))
    h = rng.uniform(0.8, 1.6)

    def pos(u, w):
        a = 2 * np.pi * u
        return np.stack([np.cos(a), np.sin(a), (w - 0.5) * h], 1) / max(1.0, h / 2 * 1.0)

    return _grid_mesh(pos, nu, nvq, True, False, chart)


def open_box(rng, n_faces, chart):
    k = max(1, int(round(math.sqrt(n_faces / 10.0))))
    dims = rng.uniform(0.5, 1.0, size=3)
    verts, tris, off = [], [], 0
    missing = int(rng.integers(0, 6))
    for face in range(6):
        if face == missing:
            continue
        axis, sign = face // 2, 1.0 if face % 2 else -1.0

        def pos(u, w, axis=axis, sign=sign):
            p = np.zeros((u.shape[0], 3))
            a1, a2 = (axis + 1) % 3, (axis + 2) % 3
            p[:, axis] = sign * 0.5
            p[:, a1] = u - 0.5
            p[:, a2] = w - 0.5
            return p

        v, t = _grid_mesh(pos, k, k, False, False, chart)
        verts.append(v * dims)
        tris.append(t + off)
        off += v.shape[0]
    return np.concatenate(verts), np.concatenate(tris)


def random_rotation(rng):
    q, r = np.linalg.qr(rng.normal(size=(3, 3)))
    q *= np.sign(np.diag(r))
    if np.linalg.det(q) < 0:
        q[:, 0] = -q[:, 0]
    return q


def add_slivers(rng, v, f, frac):
    """Replace a fraction of faces (a,b,c) by (a,b,c') with c' within 1e-6 of edge ab."""
    nf = f.shape[0]
    k = int(round(frac * nf))
    if k == 0:
        return v, f
    sel = rng.choice(nf, size=k, replace=False)
    a, b = v[f[sel, 0]], v[f[sel, 1]]
    t = rng.uniform(0.2, 0.8, size=(k, 1))
    d = rng.normal(size=(k, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    cp = a + t * (b - a) + 1e-6 * d
    new_ids = np.arange(v.shape[0], v.shape[0] + k)
    v = np.concatenate([v, cp])
    f = f.copy()
    f[sel, 2] = new_ids
    return v, f


def _place(rng, v, scale, lo=-0.5, hi=0.5):
    v = v @ random_rotation(rng).T
    ext = np.abs(v).max() * scale
    c = rng.uniform(lo + ext, hi - ext, size=3) if hi - lo > 2 * ext else np.full(3, (lo + hi) / 2)
    return v * scale + c


# --------------------------------------------------------------------------- workloads
def ico_cap(seed: int = 0) -> Workload:
    rng = np.random.default_rng(seed)
    v, f = icosphere(4)
    v = v * 0.4
    v = v + rng.normal(0.0, 1e-3, size=v.shape)
    axis = rng.normal(size=3)
    axis /= np.linalg.norm(axis)
    cent = v[f].mean(axis=1)
    cosang = (cent @ axis) / np.linalg.norm(cent, axis=1)
    keep = cosang < math.cos(math.radians(20.0))
    f = f[keep]
    return Workload("ico_cap", v.astype(np.float32), f.astype(np.int64), 64, UNIT_AABB,
                    meta={"config": "icosphere L4, r=0.4, 20 deg cap removed, grid 64"})


def _primitive_soup(rng, n_prims, faces_total, aabb_lo=-0.5, aabb_hi=0.5):
    per = faces_total / n_prims
    kinds = [torus, open_cylinder, open_box, None]
    verts, tris, off = [], [], 0
    for p in range(n_prims):
        kind = kinds[p % 4]
        chart = 3 if (p % 7) else 2
        if kind is None:
            level = max(0, min(6, int(round(math.log(max(per, 20) / 20.0, 4)))))
            v, t = icosphere(level)
        else:
            v, t = kind(rng, per, chart)
        scale = rng.uniform(0.05, 0.3)
        v = _place(rng, v, scale, aabb_lo, aabb_hi)
        verts.append(v)
        tris.append(t + off)
        off += v.shape[0]
    return np.concatenate(verts), np.concatenate(tris)


def primitives(seed: int = 1, faces_total: int = 290_000) -> Workload:
    rng = np.random.default_rng(seed)
    v, f = _primitive_soup(rng, 48, faces_total)
    v, f = add_slivers(rng, v, f, 0.01)
    return Workload("primitives", v.astype(np.float32), f.astype(np.int64), 512, UNIT_AABB,
                    meta={"config": "48 primitives, ~280k faces, 1% slivers, grid 512"})


def subdivided(seed: int = 1, target_faces: int = 10_300_000, grid_size: int = 512) -> Workload:
    base = primitives(seed)
    rng = np.random.default_rng(seed + 1000)
    v = base.vertices.astype(np.float64)
    f = base.faces
    v, f = _subdivide_all(v, f)
    v, f = _subdivide_all(v, f)
    extra = max(0, (target_faces - f.shape[0]) // 3)
    extra = min(extra, f.shape[0])
    sel = np.zeros(f.shape[0], dtype=bool)
    sel[rng.choice(f.shape[0], size=extra, replace=False)] = True
    v2, f2 = _subdivide_all(v, f[sel])
    f = np.concatenate([f[~sel], f2])
    v = v2
    return Workload("subdivided", v.astype(np.float32), f.astype(np.int64), grid_size, UNIT_AABB,
                    meta={"config": f"primitives x2 midpoint subdivision + {extra} faces once more, grid {grid_size}"})


def sheets(seed: int = 3, n_sheets: int = 2000, n_creases: int = 1000, grid_size: int = 1024) -> Workload:
    rng = np.random.default_rng(seed)
    vs = 1.0 / grid_size
    verts, tris, off = [], [], 0
    # stacks of near-coplanar sheets, spacing 0.3 voxel, normals perturbed by ~1e-5 rad
    n_stacks = 20
    per_stack = n_sheets // n_stacks
    for s in range(n_stacks):
        rot = random_rotation(rng)
        size = rng.uniform(0.04, 0.08)
        height = per_stack * 0.3 * vs
        ext = 0.5 * math.sqrt(2 * size * size + height * height) + 2 * vs
        centre = rng.uniform(-0.5 + ext, 0.5 - ext, size=3)
        for k in range(per_stack):
            # 6 x 7 quads = 84 triangles a sheet: 2000 sheets and 1000 creases of 32 give 200k faces
            v, t = _grid_mesh(lambda u, w: np.stack([u - 0.5, w - 0.5, np.zeros_like(u)], 1), 6, 7, False, False, 64)
            ang = 1e-5 * rng.normal(size=3)
            small = np.array([[1, -ang[2], ang[1]], [ang[2], 1, -ang[0]], [-ang[1], ang[0], 1]])
            v = (v * size) @ small.T
            v[:, 2] += (k - per_stack / 2) * 0.3 * vs
            v = v @ rot.T + centre
            verts.append(v)
            tris.append(t + off)
            off += v.shape[0]
    # creases: two strips meeting along a shared edge at a dihedral angle in [1,179] deg
    for c in range(n_creases):
        ang = math.radians(rng.uniform(1.0, 179.0))
        size = rng.uniform(0.01, 0.03)
        nq = 8
        u = np.linspace(0, 1, nq + 1)
        a = np.stack([np.zeros_like(u), u, np.zeros_like(u)], 1)
        b = np.stack([np.full_like(u, 1.0), u, np.zeros_like(u)], 1)
        cc = np.stack([np.full_like(u, math.cos(ang)), u, np.full_like(u, math.sin(ang))], 1)
        v = np.concatenate([a, b, cc]) * size
        ids = np.arange(nq)
        t = np.concatenate([
            np.stack([ids, ids + nq + 1, ids + nq + 2], 1), np.stack([ids, ids + nq + 2, ids + 1], 1),
            np.stack([ids, ids + 2 * (nq + 1) + 1, ids + 2 * (nq + 1)], 1), np.stack([ids, ids + 1, ids + 2 * (nq + 1) + 1], 1)])
        v = _place(rng, v - v.mean(0), 1.0)
        verts.append(v)
        tris.append(t + off)
        off += v.shape[0]
    v = np.concatenate(verts)
    f = np.concatenate(tris)
    v, f = add_slivers(rng, v, f, 0.2)
    return Workload("sheets", v.astype(np.float32), f.astype(np.int64), grid_size, UNIT_AABB,
                    meta={"config": f"{n_sheets} near-coplanar sheets (0.3 voxel spacing), {n_creases} creases, 20% slivers, grid {grid_size}"})


def lowpoly(seed: int = 5, faces_total: int = 1_200, grid_size: int = 512) -> Workload:
    """A low-poly soup of primitives on a fine grid: about a thousand triangles,
    most spanning thousands of cells per projection and hundreds of bricks,
    so the large-triangle paths do nearly all the work."""
    rng = np.random.default_rng(seed)
    v, f = _primitive_soup(rng, 16, faces_total)
    v, f = add_slivers(rng, v, f, 0.01)
    lo, hi = v.min(0), v.max(0)
    pad = (hi - lo) / (grid_size - 1) * 0.5
    aabb = [list(map(float, lo - pad)), list(map(float, hi + pad))]
    return Workload("lowpoly", v.astype(np.float32), f.astype(np.int64), grid_size, aabb,
                    meta={"config": f"16 primitives, {f.shape[0]} faces, grid {grid_size}, per-mesh aabb"})


def batch(seed: int = 4, n_meshes: int = 256, f_lo: int = 1_000, f_hi: int = 500_000,
          grids=(64, 128, 256, 512)) -> List[Workload]:
    rng = np.random.default_rng(seed)
    out = []
    for m in range(n_meshes):
        nf = int(round(math.exp(rng.uniform(math.log(f_lo), math.log(f_hi)))))
        n_prims = int(rng.integers(4, 49))
        v, f = _primitive_soup(rng, n_prims, nf)
        v, f = add_slivers(rng, v, f, 0.01)
        g = int(rng.choice(grids))
        lo, hi = v.min(0), v.max(0)
        pad = (hi - lo) / (g - 1) * 0.5
        aabb = [list(map(float, lo - pad)), list(map(float, hi + pad))]
        out.append(Workload(f"batch{m}", v.astype(np.float32), f.astype(np.int64), g, aabb,
                            meta={"config": f"batch mesh {m}: {f.shape[0]} faces, grid {g}"}))
    return out


def small_cases() -> List[Workload]:
    """Hand-built edge cases: exact dyadic triangles on grid planes, slivers,
    an open boundary, a non-manifold edge, vertices outside the aabb, empty mesh."""
    cases = []
    g = 16
    aabb = [[0.0, 0.0, 0.0], [1.0, 1.0, 1.0]]
    # single axis-aligned triangle lying exactly on grid planes
    v = np.array([[0.25, 0.25, 0.5], [0.75, 0.25, 0.5], [0.25, 0.75, 0.5]], np.float32)
    cases.append(Workload("on_plane", v, np.array([[0, 1, 2]], np.int64), g, aabb))
    # triangle with vertices exactly on voxel corners, tilted
    v = np.array([[0.125, 0.125, 0.125], [0.875, 0.25, 0.5], [0.25, 0.875, 0.75]], np.float32)
    cases.append(Workload("dyadic_tilted", v, np.array([[0, 1, 2]], np.int64), g, aabb))
    # sliver: third vertex 1e-6 from the opposite edge
    v = np.array([[0.1, 0.2, 0.3], [0.9, 0.7, 0.6], [0.5, 0.45 + 1e-6, 0.45]], np.float32)
    cases.append(Workload("sliver", v, np.array([[0, 1, 2]], np.int64), g, aabb))
    # non-manifold edge: three faces share edge (0,1)
    v = np.array([[0.2, 0.5, 0.5], [0.8, 0.5, 0.5], [0.5, 0.9, 0.5], [0.5, 0.1, 0.55], [0.5, 0.5, 0.9]], np.float32)
    cases.append(Workload("nonmanifold", v, np.array([[0, 1, 2], [1, 0, 3], [0, 1, 4]], np.int64), g, aabb))
    # open quad strip (boundary everywhere) partly outside the aabb
    v = np.array([[-0.2, 0.3, 0.4], [1.2, 0.35, 0.45], [-0.1, 0.8, 0.6], [1.1, 0.85, 0.5]], np.float32)
    cases.append(Workload("outside_aabb", v, np.array([[0, 1, 2], [2, 1, 3]], np.int64), g, aabb))
    # degenerate face (repeated index) next to a normal one
    v = np.array([[0.3, 0.3, 0.3], [0.7, 0.4, 0.35], [0.4, 0.7, 0.6]], np.float32)
    cases.append(Workload("degenerate", v, np.array([[0, 0, 1], [0, 1, 2]], np.int64), g, aabb))
    # non-cubic grid with a non power-of-two voxel size
    rng = np.random.default_rng(7)
    v, f = icosphere(2)
    v = (v * 0.35 + 0.5 + rng.normal(0, 1e-3, v.shape)).astype(np.float32)
    cases.append(Workload("ico_anisotropic", v, f.astype(np.int64), [24, 40, 33], [[0.02, 0.0, 0.05], [0.97, 1.0, 0.99]]))
    # empty mesh
    cases.append(Workload("empty", np.zeros((0, 3), np.float32), np.zeros((0, 3), np.int64), g, aabb))
    return cases
