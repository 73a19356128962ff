"""Generates tests/golden/fma_probe.npz: per-triangle surface hit sets of the
reference's own CUDA kernels (oracle/_ref/libvoxref.so) for isolated
triangles whose vertices sit exactly on voxel centres, cell faces and cell
corners.  At those ties the result of the conservative triangle/box tests
(src/voxelizer.cu:2633-2942, 3306-4119) depends on which multiply-adds nvcc
fused, so these sets pin the oracle's contraction model site by site.

Each scene holds up to 253 probe triangles, each alone in its own 10-voxel
cell with a unique material (LongNode keeps 8-bit materials), plus two tiny
anchor triangles (material 255) that fix the bounding box.  The output of a
scene is the list of (node index, material) pairs with a non-zero material.

Usage (needs a GPU):  python tests/golden/make_fma_probe.py --out tests/golden
"""

from __future__ import annotations

import argparse
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from voxelizer_b200.scenes import Mesh  # noqa: E402

# (cube length, bounding-box minimum) per scene family.
FAMILIES = [(1.0 / 128.0, 0.1), (0.8 / 100.0, 0.1), (0.0123, -0.37)]
CELL = 10          # voxels per probe cell
SLOTS = 10         # cells per axis
PER_SCENE = 253


def probe_scene(seed, family):
    d, lo = FAMILIES[family]
    rng = np.random.default_rng(seed)
    span = CELL * SLOTS * d
    verts, mats = [], []
    # Anchors: a tiny triangle at each extreme corner of the bounding box.
    a0 = np.array([[lo, lo, lo], [lo + 0.2 * d, lo, lo], [lo, lo + 0.2 * d, lo]])
    hi = lo + span + 2 * d
    a1 = np.array([[hi, hi, hi], [hi - 0.2 * d, hi, hi], [hi, hi - 0.2 * d, hi]])
    verts += [a0, a1]
    mats += [255, 255]
    cells = rng.permutation(SLOTS ** 3)[:PER_SCENE]
    lo32 = np.float32(lo)
    for k, cell in enumerate(cells):
        cz, cy, cx = cell // (SLOTS * SLOTS), (cell // SLOTS) % SLOTS, cell % SLOTS
        base = np.array([cx, cy, cz]) * CELL + 3
        kind = rng.integers(0, 6)
        # Offsets in half-voxel steps: 0 is a voxel centre, 1 a cell face.
        off = rng.integers(-2, 7, size=(3, 3)) / 2.0
        if kind == 1:      # flat in x (2D / 1D classes)
            off[:, 0] = off[0, 0]
        elif kind == 2:    # flat in y
            off[:, 1] = off[0, 1]
        elif kind == 3:    # flat in z
            off[:, 2] = off[0, 2]
        elif kind == 4:    # thin: two coordinates shared
            ax = rng.integers(0, 3)
            for a in range(3):
                if a != ax:
                    off[:, a] = off[0, a]
            off[2, ax] = off[1, ax] + 0.5
        pos = np.float64(lo32) + (base[None, :] + off) * d
        verts.append(pos)
        mats.append(k + 1)
    v = np.concatenate(verts).astype(np.float32)
    idx = np.arange(v.shape[0], dtype=np.uint32).reshape(-1, 3)
    return Mesh(v, idx, np.array(mats, np.uint8), 256, f"probe{family}_{seed}"), d


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--scenes", type=int, default=12)
    args = ap.parse_args()
    import make_golden as G
    f = G.load_ref()
    os.makedirs(args.out, exist_ok=True)
    recs = {}
    for s in range(args.scenes):
        fam = s % len(FAMILIES)
        m, d = probe_scene(1000 + s, fam)
        dims = (ctypes.c_uint32 * 3)()
        vs = (ctypes.c_uint32 * 3)(1024, 512, 512)
        ms = (ctypes.c_uint32 * 3)(512, 512, 512)
        args_ = [1, 1, 1, 1, 0, float(d), vs, ms, m.vertices.ctypes.data, m.n_vertices, m.indices.ctypes.data,
                 m.n_triangles, m.materials.ctypes.data, 256]
        rc = f(*args_, None, 0, dims, None)
        assert rc == 0, rc
        n = int(dims[0]) * int(dims[1]) * int(dims[2])
        out = np.empty(n, np.uint16)
        rc = f(*args_, out.ctypes.data, out.nbytes, dims, None)
        assert rc == 0, rc
        mat = (out >> 8).astype(np.uint8)
        nz = np.nonzero(mat)[0].astype(np.uint32)
        recs[f"s{s}_idx"] = nz
        recs[f"s{s}_mat"] = mat[nz]
        recs[f"s{s}_dims"] = np.array([int(dims[0]), int(dims[1]), int(dims[2])], np.uint32)
        print(f"scene {s}: family {fam}, dims {tuple(dims)}, {nz.size} surface nodes", flush=True)
    np.savez_compressed(os.path.join(args.out, "fma_probe.npz"), **recs)


if __name__ == "__main__":
    main()
