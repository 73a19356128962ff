"""Golden-vector cases: each names a seeded input mesh and one call of the
reference API (``Voxelizer<Node>::voxelizeToRAM`` / ``voxelizeToNodesToRAM``,
include/voxelizer.h:727-782).  ``make_golden.py`` runs every case through the
reference's own CUDA kernels (oracle/_ref) on a B200 and stores the output;
the tests rebuild the same inputs from this file and compare.

Node types follow include/node_types.h: 0 ShortNode, 1 LongNode,
2 PartialNode, 3 ShortFCCNode, 4 LongFCCNode.
"""

from __future__ import annotations

import hashlib

import numpy as np

from voxelizer_b200 import scenes

SHORT, LONG, PARTIAL, SHORT_FCC, LONG_FCC = range(5)
NODE_BYTES = {SHORT: 1, LONG: 2, PARTIAL: 8, SHORT_FCC: 2, LONG_FCC: 4}
FCC_A = 4.0 ** (1.0 / 3.0) / 128.0  # FCC cell edge with the node density of a 1/128 cubic grid

DEFAULT_VOX = (1024, 512, 512)
DEFAULT_MAT = (512, 512, 512)


def _ico4(level=4):
    v, f = scenes.icosphere(level, 0.4, (0.5, 0.5, 0.5))
    return scenes.Mesh(v, f, np.ones(f.shape[0], np.uint8), 2, f"ico{level}")


def _ico_mixed(level=3):
    v, f = scenes.icosphere(level, 0.4, (0.5, 0.5, 0.5))
    m = (1 + np.arange(f.shape[0]) % 7).astype(np.uint8)   # tests/src/main.cpp:1550-1561
    return scenes.Mesh(v, f, m, 8, f"ico{level}_mixed")


def _torus():
    rng = np.random.default_rng(7)
    v, f = scenes.torus(64, 32)
    v = scenes.transform(v, scenes.random_rotation(rng), 0.45, (0.5, 0.5, 0.5))
    return scenes.Mesh(v, f, np.full(f.shape[0], 3, np.uint8), 4, "torus64x32")


def _stress(cube=1.0 / 128.0, n_sl=2000, n_sn=1000, seed=1):
    return scenes.stress_scene(n_sl, n_sn, seed=seed, level=4, cube_length=cube)


def _room_lite():
    return scenes.room_scene(n_objects=12, seed=3, target=None, scale_range=(0.3, 0.8),
                             clearance=2.0 * 10.0 / 159.0)


def _room_full():
    return scenes.room_scene()


def _elong(level=4):
    v, f = scenes.icosphere(level, 0.4, (0.5, 0.5, 0.5))
    v = scenes.transform(v, None, (16.0, 1.0, 1.0))
    return scenes.Mesh(v, f, np.ones(f.shape[0], np.uint8), 2, f"elong_ico{level}")


MESHES = {
    "ico4": _ico4,
    "ico3_mixed": _ico_mixed,
    "torus": _torus,
    "stress": _stress,
    "stress_fcc": lambda: _stress(cube=FCC_A, seed=2),
    "room_lite": _room_lite,
    "room_full": _room_full,
    "elong4": _elong,
    "stress_full_fcc": lambda: scenes.stress_scene(10_000, 5_000, seed=4, level=4, cube_length=FCC_A),
}

_MESH_CACHE: dict = {}


def mesh(name):
    if name not in _MESH_CACHE:
        _MESH_CACHE[name] = MESHES[name]()
    return _MESH_CACHE[name]


def case(name, mesh, node_type, nodes, materials, size, vox=DEFAULT_VOX, mat=DEFAULT_MAT, store="full",
         strict_mats=True, space=None):
    """``size`` is an int (maxDimension) or a float (cubeLength).
    ``store`` is "full" (array kept) or "digest" (SHA-256 and counts only).
    ``strict_mats`` is False where triangles of different materials touch the
    same voxel, so that the reference's plain-store race (src/voxelizer.cu:2988)
    makes its material bytes nondeterministic there.
    ``space`` voxelizes one device space instead of the whole grid:
    ("slice", direction, s) the slice s (1-based, padding row 0) along y (1)
    or z (2); ("part", dev_y, dev_z, k) partition k (y fastest) of devConfig
    (dev_y, dev_z)."""
    return dict(name=name, mesh=mesh, node_type=node_type, nodes=int(nodes), materials=int(materials),
                by_cube=isinstance(size, float), size=size, vox=tuple(vox), mat=tuple(mat), store=store,
                strict_mats=strict_mats, space=tuple(space) if space else None)


def split_parts(length, parts):
    """splitResolutionByNrOfParts along one axis: floor division, the
    remainder to the first part (src/host_side.cpp:3025-3105)."""
    out, prev = [None] * parts, length
    for i in range(parts, 0, -1):
        lo = prev - prev // i
        out[i - 1] = (lo, prev)
        prev = lo
    return out


def partition(c, res_y, res_z):
    """(y0, y1, z0, z1) of a case's device space for a grid of res_y x res_z
    voxel rows; None for the whole grid."""
    sp = c.get("space")
    if not sp:
        return None
    if sp[0] == "slice":
        # direction 0 (x) slices the turned grid along its y (res_y, res_z of
        # the turned grid then)
        _, direction, s = sp
        n = res_z if direction == 2 else res_y
        s0 = 0 if (s == 0 or s > n) else s - 1   # sliceOOB voxelizes row 0 (and zeroes the result)
        return (0, res_y, s0, s0 + 1) if direction == 2 else (s0, s0 + 1, 0, res_z)
    _, dy, dz, k = sp
    ys, zs = split_parts(res_y, dy), split_parts(res_z, dz)
    y, z = k % dy, k // dy
    return (ys[y][0], ys[y][1], zs[z][0], zs[z][1])


def slice_oob(c, res_y, res_z):
    sp = c.get("space")
    if not sp or sp[0] != "slice":
        return False
    n = res_z if sp[1] == 2 else res_y
    return sp[2] == 0 or sp[2] > n


def turned(c):
    """True for slices along x, which voxelize the mesh turned about z."""
    sp = c.get("space")
    return bool(sp) and sp[0] == "slice" and sp[1] == 0


CASES = [
    # Plain single mesh (icosphere L4, 1/128): nodes and bit array.
    case("ico4_short_mat", "ico4", SHORT, 1, 1, 1.0 / 128.0),
    case("ico4_short_nomat", "ico4", SHORT, 1, 0, 1.0 / 128.0),
    case("ico4_bits", "ico4", SHORT, 0, 0, 1.0 / 128.0),
    case("ico4_long_md100", "ico4", LONG, 1, 1, 100),
    # Many small yz / x / material splits: tile straddling and split-ordered pruning.
    case("ico3_long_splits", "ico3_mixed", LONG, 1, 1, 90, vox=(64, 16, 16), mat=(16, 16, 16), strict_mats=False),
    case("ico3_bits_splits", "ico3_mixed", LONG, 0, 0, 90, vox=(64, 16, 16)),
    case("torus_long", "torus", LONG, 1, 1, 120),
    case("torus_short_splits", "torus", SHORT, 1, 1, 120, vox=(32, 24, 40), mat=(40, 24, 32)),
    # Degeneracy stress: slivers and snapped vertices (ties everywhere).
    case("stress_bits", "stress", SHORT, 0, 0, 1.0 / 128.0),
    case("stress_short_mat", "stress", SHORT, 1, 1, 1.0 / 128.0, strict_mats=False),
    case("stress_long_nomat", "stress", LONG, 1, 0, 1.0 / 128.0),
    case("stress_long_splits", "stress", LONG, 1, 1, 1.0 / 128.0, vox=(96, 40, 40), mat=(40, 40, 40),
         strict_mats=False),
    # FCC lattices.
    case("ico4_sfcc_mat", "ico4", SHORT_FCC, 1, 1, FCC_A),
    case("ico4_lfcc_nomat", "ico4", LONG_FCC, 1, 0, FCC_A),
    case("stress_sfcc_mat", "stress_fcc", SHORT_FCC, 1, 1, FCC_A, strict_mats=False),
    case("stress_lfcc_mat", "stress_fcc", LONG_FCC, 1, 1, FCC_A, vox=(64, 32, 32), mat=(32, 32, 32),
         strict_mats=False),
    # Room scene, reduced and full size.
    case("room_lite_long", "room_lite", LONG, 1, 1, 160),
    case("room_lite_bits", "room_lite", LONG, 0, 0, 160),
    # Elongated grid: several x splits.
    case("elong4_bits", "elong4", SHORT, 0, 0, 2048),
    case("elong4_long_nomat", "elong4", LONG, 1, 0, 1024),
    # Full-size configurations (digest only).
    case("room_full_long", "room_full", LONG, 1, 1, 1024, store="digest"),
    case("room_full_bits", "room_full", LONG, 0, 0, 1024, store="digest"),
    case("elong4_4096_long", "elong4", LONG, 1, 0, 4096, store="digest"),
    case("stress_full_sfcc", "stress_full_fcc", SHORT_FCC, 1, 1, FCC_A, strict_mats=False),
    # PartialNode without and with materials (the surface ratio depends on
    # which racing triangle wrote last).
    case("ico4_partial_nomat", "ico4", PARTIAL, 1, 0, 1.0 / 64.0),
    case("ico4_partial_mat", "ico4", PARTIAL, 1, 1, 1.0 / 64.0, strict_mats=False),
    case("torus_partial_mat", "torus", PARTIAL, 1, 1, 96, strict_mats=False),
    case("stress_partial_mat", "stress", PARTIAL, 1, 1, 1.0 / 96.0, mat=(48, 48, 48), strict_mats=False),
    # Device spaces: slices (voxelizeSlice) and devConfig partitions.
    case("torus_long_slice_y_mid", "torus", LONG, 1, 1, 120, space=("slice", 1, 50)),
    case("torus_long_slice_y_first", "torus", LONG, 1, 1, 120, space=("slice", 1, 1)),
    case("torus_long_slice_y_last", "torus", LONG, 1, 1, 120, space=("slice", 1, 120)),
    case("torus_short_slice_z_mid", "torus", SHORT, 1, 1, 120, space=("slice", 2, 20)),
    case("ico3_long_slice_z_splits", "ico3_mixed", LONG, 1, 1, 90, vox=(64, 16, 16), mat=(16, 16, 16),
         strict_mats=False, space=("slice", 2, 40)),
    case("torus_long_slice_oob", "torus", LONG, 1, 1, 120, space=("slice", 1, 0)),
    case("room_lite_long_part22_0", "room_lite", LONG, 1, 1, 160, space=("part", 2, 2, 0)),
    case("room_lite_long_part22_1", "room_lite", LONG, 1, 1, 160, space=("part", 2, 2, 1)),
    case("room_lite_long_part22_2", "room_lite", LONG, 1, 1, 160, space=("part", 2, 2, 2)),
    case("room_lite_long_part22_3", "room_lite", LONG, 1, 1, 160, space=("part", 2, 2, 3)),
    case("ico4_partial_part31_1", "ico4", PARTIAL, 1, 1, 1.0 / 64.0, strict_mats=False, space=("part", 3, 1, 1)),
    case("room_lite_bits_part13_1", "room_lite", LONG, 0, 0, 160, space=("part", 1, 3, 1)),
    # FCC device spaces: y / z slices and devConfig partitions.
    case("ico4_sfcc_slice_y_mid", "ico4", SHORT_FCC, 1, 1, FCC_A, space=("slice", 1, 30)),
    case("ico4_lfcc_slice_z_mid", "ico4", LONG_FCC, 1, 0, FCC_A, space=("slice", 2, 33)),
    case("ico4_sfcc_slice_oob", "ico4", SHORT_FCC, 1, 1, FCC_A, space=("slice", 2, 0)),
    case("ico4_sfcc_part22_0", "ico4", SHORT_FCC, 1, 1, FCC_A, space=("part", 2, 2, 0)),
    case("ico4_sfcc_part22_3", "ico4", SHORT_FCC, 1, 1, FCC_A, space=("part", 2, 2, 3)),
    case("stress_lfcc_part31_1", "stress_fcc", LONG_FCC, 1, 1, FCC_A, vox=(64, 32, 32), mat=(32, 32, 32),
         strict_mats=False, space=("part", 3, 1, 1)),
    # Slices along x: the mesh turned about z, sliced along the turned y.
    case("torus_long_slice_x_mid", "torus", LONG, 1, 1, 120, space=("slice", 0, 40)),
    case("torus_short_slice_x_first", "torus", SHORT, 1, 1, 120, space=("slice", 0, 1)),
    case("ico3_long_slice_x_splits", "ico3_mixed", LONG, 1, 1, 90, vox=(64, 16, 16), mat=(16, 16, 16),
         strict_mats=False, space=("slice", 0, 45)),
    case("torus_partial_slice_x", "torus", PARTIAL, 1, 1, 96, strict_mats=False, space=("slice", 0, 30)),
    case("torus_long_slice_x_oob", "torus", LONG, 1, 1, 120, space=("slice", 0, 500)),
    case("ico4_sfcc_slice_x_mid", "ico4", SHORT_FCC, 1, 1, FCC_A, space=("slice", 0, 30)),
    case("ico4_lfcc_slice_x_first", "ico4", LONG_FCC, 1, 0, FCC_A, space=("slice", 0, 1)),
    case("stress_sfcc_slice_x", "stress_fcc", SHORT_FCC, 1, 1, FCC_A, vox=(64, 32, 32), mat=(32, 32, 32),
         strict_mats=False, space=("slice", 0, 40)),
]

BY_NAME = {c["name"]: c for c in CASES}


def mesh_digest(m):
    h = hashlib.sha256()
    h.update(m.vertices.tobytes())
    h.update(m.indices.tobytes())
    if m.materials is not None:
        h.update(m.materials.tobytes())
    return h.hexdigest()


def out_dtype(c):
    if not c["nodes"]:
        return np.uint32
    return {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}[NODE_BYTES[c["node_type"]]]
