"""Generates tests/golden/fma_probe_nt{0..4}.npz: the surface nodes of the
reference's own CUDA kernels (oracle/_ref/libvoxref.so) for isolated
triangles whose vertices sit exactly on voxel centres, cell faces and cell
corners, one file per node type (include/node_types.h: 0 ShortNode,
1 LongNode, 2 PartialNode, 3 ShortFCCNode, 4 LongFCCNode).  At those ties the
result of the conservative triangle/box tests (src/voxelizer.cu:2633-2942,
3306-4119) depends on which multiply-adds nvcc fused, and the fused forms
differ between the node types' instantiations of the class kernels, so these
sets pin the oracle's contraction model site by site and per node type.

Each scene holds up to 253 probe triangles, each alone in its own 10-voxel
cell, plus two tiny anchor triangles that fix the bounding box; every
triangle has material 1.  The stored output of a scene is the sorted list of
node indices whose material is non-zero (the surface nodes).

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
SCENES = 30
NODE_BYTES = {0: 1, 1: 2, 2: 8, 3: 2, 4: 4}
MAT_SHIFT = {0: 5, 1: 8, 2: 8, 3: 12, 4: 16}
MAT_MASK = {0: 7, 1: 255, 2: 255, 3: 15, 4: 255}


def probe_scene(seed, family):
    """The probe mesh of one scene: anchors, then one triangle per cell."""
    d, lo = FAMILIES[family]
    rng = np.random.default_rng(seed)
    span = CELL * SLOTS * d
    verts = []
    # Anchors: a tiny triangle at each extreme corner of the bounding box.
    a0 = np.array([[lo, lo, lo], [lo + 0.2 * d, lo, lo], [lo, lo + 0.2 * d, lo]])
    hi = lo + span + 2 * d
    a1 = np.array([[hi, hi, hi], [hi - 0.2 * d, hi, hi], [hi, hi - 0.2 * d, hi]])
    verts += [a0, a1]
    cells = rng.permutation(SLOTS ** 3)[:PER_SCENE]
    lo32 = np.float32(lo)
    for cell in cells:
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
    v = np.concatenate(verts).astype(np.float32)
    idx = np.arange(v.shape[0], dtype=np.uint32).reshape(-1, 3)
    mats = np.ones(idx.shape[0], np.uint8)
    return Mesh(v, idx, mats, 2, f"probe{family}_{seed}"), d


def scene(s):
    """Scene s of the probe set: (mesh, cube length)."""
    return probe_scene(1000 + s, s % len(FAMILIES))


def surface_nodes(node_type, out):
    """Indices of the nodes whose material field is non-zero."""
    a = out.astype(np.uint64)
    mat = (a >> np.uint64(MAT_SHIFT[node_type])) & np.uint64(MAT_MASK[node_type])
    return np.nonzero(mat)[0].astype(np.uint32)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--scenes", type=int, default=SCENES)
    ap.add_argument("--node-types", default="0,1,2,3,4")
    args = ap.parse_args()
    import make_golden as G
    f = G.load_ref()
    os.makedirs(args.out, exist_ok=True)
    dt = {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}
    for nt in [int(t) for t in args.node_types.split(",")]:
        recs = {}
        for s in range(args.scenes):
            m, d = scene(s)
            dims = (ctypes.c_uint32 * 3)()
            vs = (ctypes.c_uint32 * 3)(1024, 512, 512)
            ms = (ctypes.c_uint32 * 3)(512, 512, 512)
            args_ = [nt, 1, 1, 1, 0, float(d), vs, ms, m.vertices.ctypes.data, m.n_vertices, m.indices.ctypes.data,
                     m.n_triangles, m.materials.ctypes.data, m.n_materials, None, 0]
            rc = f(*args_, None, 0, dims, None)
            assert rc == 0, (rc, f.last_error())
            n = int(dims[0]) * int(dims[1]) * int(dims[2])
            out = np.empty(n, dt[NODE_BYTES[nt]])
            rc = f(*args_, out.ctypes.data, out.nbytes, dims, None)
            assert rc == 0, (rc, f.last_error())
            recs[f"s{s}_idx"] = surface_nodes(nt, out)
            recs[f"s{s}_dims"] = np.array([int(dims[0]), int(dims[1]), int(dims[2])], np.uint32)
            print(f"node type {nt} scene {s}: dims {tuple(dims)}, {recs[f's{s}_idx'].size} surface nodes", flush=True)
        np.savez_compressed(os.path.join(args.out, f"fma_probe_nt{nt}.npz"), **recs)


if __name__ == "__main__":
    main()
