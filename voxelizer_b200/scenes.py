"""Seeded synthetic meshes for tests and benchmarks.

Every generator returns ``(vertices, indices)`` as contiguous ``float32 [V,3]``
and ``uint32 [T,3]`` arrays (the layout ``vox::Voxelizer``'s constructor takes:
three floats per vertex, three indices per triangle), plus per-triangle
``uint8`` materials where a scene defines them.  All randomness comes from
``numpy.random.default_rng(seed)`` so a scene is a pure function of its
arguments.

Scenes:

* ``icosphere(level)``       closed subdivided icosahedron, 20*4**level triangles
* ``torus(u, v)``            closed torus, 2*u*v triangles
* ``room_scene(...)``        inward box shell holding non-overlapping rotated
                             icospheres and tori with ≥2-voxel clearance
* ``stress_scene(...)``      icosphere + sliver triangles + triangles whose
                             vertices sit exactly on voxel centres / cell faces
* ``batch_mix(...)``         many independent meshes with log-uniform sizes
"""

from __future__ import annotations

import math

import numpy as np

__all__ = [
    "icosphere", "torus", "room_scene", "stress_scene", "batch_mix", "transform",
    "random_rotation", "Mesh",
]


class Mesh:
    """A triangle mesh plus optional per-triangle materials."""

    def __init__(self, vertices, indices, materials=None, n_materials=0, name=""):
        self.vertices = np.ascontiguousarray(vertices, dtype=np.float32).reshape(-1, 3)
        self.indices = np.ascontiguousarray(indices, dtype=np.uint32).reshape(-1, 3)
        self.materials = None if materials is None else np.ascontiguousarray(materials, dtype=np.uint8)
        self.n_materials = int(n_materials)
        self.name = name

    @property
    def n_vertices(self):
        return int(self.vertices.shape[0])

    @property
    def n_triangles(self):
        return int(self.indices.shape[0])

    def __repr__(self):
        return f"Mesh({self.name!r}, V={self.n_vertices}, T={self.n_triangles})"


def _merge(parts):
    verts, idx, mats = [], [], []
    off = 0
    for v, i, m in parts:
        verts.append(v)
        idx.append(i + off)
        mats.append(m)
        off += v.shape[0]
    return (np.concatenate(verts).astype(np.float32), np.concatenate(idx).astype(np.uint32),
            np.concatenate(mats).astype(np.uint8))


def icosphere(level: int, radius: float = 1.0, center=(0.0, 0.0, 0.0)):
    """Closed icosphere with 20*4**level triangles (vertices in float32)."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = np.array([(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t),
                  (0, -1, -t), (0, 1, -t), (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)],
                 dtype=np.float64)
    f = np.array([(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
                  (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
                  (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)], dtype=np.int64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    for _ in range(level):
        # Split every edge once: midpoints keyed by the sorted vertex pair.
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        e.sort(axis=1)
        key = e[:, 0] * (v.shape[0] + 1) + e[:, 1]
        uniq, inv = np.unique(key, return_inverse=True)
        a = uniq // (v.shape[0] + 1)
        b = uniq % (v.shape[0] + 1)
        mid = v[a] + v[b]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        m = inv.reshape(3, -1) + v.shape[0]
        m01, m12, m20 = m[0], m[1], m[2]
        v = np.concatenate([v, mid])
        f = np.concatenate([
            np.stack([f[:, 0], m01, m20], 1), np.stack([f[:, 1], m12, m01], 1),
            np.stack([f[:, 2], m20, m12], 1), np.stack([m01, m12, m20], 1)])
    v = v * radius + np.asarray(center, dtype=np.float64)
    return v.astype(np.float32), f.astype(np.uint32)


def torus(u: int, v: int, major: float = 0.7, minor: float = 0.3, center=(0.0, 0.0, 0.0)):
    """Closed torus around the z axis with 2*u*v triangles."""
    i = np.arange(u)[:, None]
    j = np.arange(v)[None, :]
    th = 2.0 * math.pi * i / u
    ph = 2.0 * math.pi * j / v
    x = (major + minor * np.cos(ph)) * np.cos(th)
    y = (major + minor * np.cos(ph)) * np.sin(th)
    z = minor * np.sin(ph) * np.ones_like(th)
    verts = np.stack([x, y, z], -1).reshape(-1, 3) + np.asarray(center, dtype=np.float64)
    a = (i * v + j)
    b = (((i + 1) % u) * v + j)
    c = (((i + 1) % u) * v + (j + 1) % v)
    d = (i * v + (j + 1) % v)
    tri = np.concatenate([np.stack([a, b, c], -1).reshape(-1, 3), np.stack([a, c, d], -1).reshape(-1, 3)])
    return verts.astype(np.float32), tri.astype(np.uint32)


def random_rotation(rng):
    """Uniform random rotation matrix (from a uniform unit quaternion)."""
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def transform(verts, rot=None, scale=1.0, offset=(0.0, 0.0, 0.0)):
    v = verts.astype(np.float64)
    if rot is not None:
        v = v @ np.asarray(rot).T
    v = v * np.asarray(scale, dtype=np.float64) + np.asarray(offset, dtype=np.float64)
    return v.astype(np.float32)


def _box_shell(lo, hi, inward=True):
    (x0, y0, z0), (x1, y1, z1) = lo, hi
    v = np.array([(x0, y0, z0), (x1, y0, z0), (x1, y1, z0), (x0, y1, z0),
                  (x0, y0, z1), (x1, y0, z1), (x1, y1, z1), (x0, y1, z1)], dtype=np.float32)
    f = np.array([(0, 2, 1), (0, 3, 2), (4, 5, 6), (4, 6, 7), (0, 1, 5), (0, 5, 4),
                  (2, 3, 7), (2, 7, 6), (1, 2, 6), (1, 6, 5), (0, 4, 7), (0, 7, 3)], dtype=np.uint32)
    if inward:
        f = f[:, ::-1].copy()
    return v, f


# Object catalogue of the room scene: (kind, parameter, triangles).
_ROOM_KINDS = [("ico", 3, 1280), ("ico", 4, 5120), ("ico", 5, 20480), ("ico", 6, 81920),
               ("torus", (64, 32), 4096), ("torus", (128, 64), 16384), ("torus", (256, 128), 65536),
               ("torus", (512, 256), 262144)]


def room_scene(n_objects=200, seed=0, size=(10.0, 7.5, 5.0), target=(950_000, 1_050_000),
               clearance=2.0 * 10.0 / 1023.0, n_materials=16, scale_range=(0.1, 0.8)):
    """Room shell [0,size] (12 inward triangles, material 1) with ``n_objects``
    closed objects, each randomly rotated, scaled and placed by rejection so
    that bounding spheres keep ``clearance`` from each other and from the walls.
    Object materials are uniform in 1..n_materials.  ``target`` bounds the
    total triangle count (``None`` disables the bound)."""
    rng = np.random.default_rng(seed)
    probs = np.array([0.36, 0.30, 0.04, 0.004, 0.26, 0.03, 0.004, 0.002])
    probs /= probs.sum()
    kinds = rng.choice(len(_ROOM_KINDS), size=n_objects, p=probs)
    if target is not None:
        lo, hi = target
        tris = np.array([_ROOM_KINDS[k][2] for k in kinds])
        order = np.argsort([_ROOM_KINDS[k][2] for k in range(len(_ROOM_KINDS))])
        for _ in range(100_000):
            total = int(tris.sum()) + 12
            if lo <= total <= hi:
                break
            pick = int(rng.integers(n_objects))
            rank = int(np.where(order == kinds[pick])[0][0])
            rank = min(rank + 1, len(order) - 1) if total < lo else max(rank - 1, 0)
            kinds[pick] = order[rank]
            tris[pick] = _ROOM_KINDS[kinds[pick]][2]
    scales = rng.uniform(*scale_range, size=n_objects)
    # Place larger objects first.
    place = np.argsort(-scales, kind="stable")
    size = np.asarray(size, dtype=np.float64)
    centers = np.zeros((n_objects, 3))
    radii = scales.copy()  # unit-radius icosphere / torus with major+minor = 1
    placed = []
    for o in place:
        r = radii[o]
        for _ in range(20000):
            c = rng.uniform(r + clearance, size - r - clearance)
            if all(np.linalg.norm(c - centers[p]) >= r + radii[p] + clearance for p in placed):
                break
        else:
            raise RuntimeError("room_scene: could not place object; lower n_objects")
        centers[o] = c
        placed.append(o)
    parts = [(*_box_shell((0, 0, 0), tuple(size)), np.ones(12, np.uint8))]
    mats = rng.integers(1, n_materials + 1, size=n_objects)
    for o in range(n_objects):
        kind, par, _ = _ROOM_KINDS[kinds[o]]
        if kind == "ico":
            v, f = icosphere(par)
        else:
            v, f = torus(par[0], par[1])
        v = transform(v, random_rotation(rng), scales[o], centers[o])
        parts.append((v, f, np.full(f.shape[0], mats[o], np.uint8)))
    v, f, m = _merge(parts)
    return Mesh(v, f, m, n_materials + 1, f"room{n_objects}_s{seed}")


def stress_scene(n_slivers=10_000, n_snapped=5_000, seed=0, level=4, cube_length=1.0 / 128.0,
                 grid_offsets=(0.0,)):
    """Closed icosphere (radius 0.4, centred in the unit cube) plus open
    degenerate-ish triangles that stress tie-breaking:

    * slivers: two long edges (length 0.05-0.6) and a width below 1e-4 of the
      length (aspect ratio > 1e4);
    * snapped: vertices placed exactly at ``min + i*d`` (voxel centres) or
      ``min + (i+1/2)*d`` (cell faces), computed in double and rounded to
      float the way the voxelizer reads them.  ``min`` is the icosphere's
      bounding-box minimum, which every added triangle stays inside so that it
      is also the mesh's.  ``grid_offsets`` adds further half-cell shifts (the
      FCC sub-lattices use d/2).
    """
    rng = np.random.default_rng(seed)
    v0, f0 = icosphere(level, 0.4, (0.5, 0.5, 0.5))
    lo = v0.astype(np.float64).min(0)
    hi = v0.astype(np.float64).max(0)
    parts = [(v0, f0, np.ones(f0.shape[0], np.uint8))]
    if n_slivers:
        a = rng.uniform(lo + 0.05, hi - 0.05, size=(n_slivers, 3))
        u = rng.normal(size=(n_slivers, 3))
        u /= np.linalg.norm(u, axis=1, keepdims=True)
        length = rng.uniform(0.05, 0.6, size=(n_slivers, 1))
        b = np.clip(a + u * length, lo, hi)
        w = rng.normal(size=(n_slivers, 3))
        w -= (w * u).sum(1, keepdims=True) * u
        w /= np.linalg.norm(w, axis=1, keepdims=True)
        width = length * rng.uniform(1e-7, 1e-4, size=(n_slivers, 1))
        c = np.clip((a + b) / 2 + w * width, lo, hi)
        v = np.stack([a, b, c], 1).reshape(-1, 3)
        parts.append((v.astype(np.float32), np.arange(3 * n_slivers, dtype=np.uint32).reshape(-1, 3),
                      np.full(n_slivers, 2, np.uint8)))
    if n_snapped:
        d = cube_length
        n = np.floor((hi - lo) / d).astype(np.int64)
        idx = rng.integers(0, np.maximum(n, 1), size=(n_snapped, 3, 3))
        half = rng.integers(0, 2, size=(n_snapped, 3, 3)) * 0.5
        off = rng.choice(np.asarray(grid_offsets, dtype=np.float64), size=(n_snapped, 3, 1))
        # Keep triangles small: second and third vertices within 3 cells of the first.
        step = rng.integers(-3, 4, size=(n_snapped, 2, 3))
        idx[:, 1:, :] = np.clip(idx[:, :1, :] + step, 0, np.maximum(n - 1, 0))
        pos = lo + (idx + half + off) * d
        pos = np.clip(pos, lo, hi)
        parts.append((pos.reshape(-1, 3).astype(np.float32),
                      np.arange(3 * n_snapped, dtype=np.uint32).reshape(-1, 3),
                      np.full(n_snapped, 3, np.uint8)))
    v, f, m = _merge(parts)
    return Mesh(v, f, m, 4, f"stress_s{seed}")


def batch_mix(n_meshes=256, seed=0, tri_range=(500, 500_000), dim_range=(32, 512), max_materials=16):
    """Independent closed meshes: triangle counts log-uniform in ``tri_range``
    (nearest icosphere/torus), non-uniform scale (1, s, s') with s, s' in
    [0.5, 1] (cubic to 2:1 boxes), ``maxDimension`` log-uniform in
    ``dim_range`` and 1..max_materials per-triangle materials.  Returns a list
    of ``(Mesh, max_dimension)``."""
    rng = np.random.default_rng(seed)
    cands = []
    for lvl in range(1, 8):
        cands.append(("ico", lvl, 20 * 4 ** lvl))
    for uu in (16, 32, 64, 128, 256, 512, 1024):
        for vv in (uu // 2, uu // 4):
            if vv >= 8:
                cands.append(("torus", (uu, vv), 2 * uu * vv))
    sizes = np.array([c[2] for c in cands], dtype=np.float64)
    out = []
    for k in range(n_meshes):
        t = math.exp(rng.uniform(math.log(tri_range[0]), math.log(tri_range[1])))
        c = cands[int(np.argmin(np.abs(np.log(sizes) - math.log(t))))]
        if c[0] == "ico":
            v, f = icosphere(c[1])
        else:
            v, f = torus(*c[1])
        s = rng.uniform(0.5, 1.0, size=2)
        v = transform(v, random_rotation(rng), (1.0, s[0], s[1]), (0.0, 0.0, 0.0))
        nm = int(rng.integers(1, max_materials + 1))
        mats = rng.integers(1, nm + 1, size=f.shape[0]).astype(np.uint8)
        md = int(round(math.exp(rng.uniform(math.log(dim_range[0]), math.log(dim_range[1])))))
        out.append((Mesh(v, f, mats, nm + 1, f"mix{k}"), md))
    return out
