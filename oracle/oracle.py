"""ctypes binding of the CPU restatement (liboracle.so, built from
vox_oracle.cpp by ``make -C oracle oracle``).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg as the checker.  The product library never uses
it.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

# Expression sites of the contraction model, in the order of ORC_S_* in
# vox_oracle.h.
SITES = ["P_BIN", "E_BIN", "D_BIN", "TN", "P_GEN", "CR_GEN", "D_GEN", "E_GEN", "B_GEN",
         "CRF_CLS", "CRF_2D", "CRF_3D", "PC_2D", "PC_3D", "PC_3DL",
         "DE_2D_YZ", "DE_2D_ZX", "DE_2D_XY", "DE_3D_YZ", "DE_3D_ZX", "DE_3D_XY",
         "OT_2D_YZ", "OT_2D_ZX", "OT_2D_XY", "OT_3D_YZ", "OT_3D_ZX", "OT_3D_XY",
         "OT_3DX_ZX", "OT_3DX_XY", "OT_3DY_XY", "OT_3DY_YZ", "OT_3DZ_YZ", "OT_3DZ_ZX",
         "DT_3DX", "DT_3DY", "DT_3DZ", "OT_2DP_YZ", "OT_2DP_ZX", "OT_2DP_XY", "UNR_2D",
         "OT_3DXP_ZX", "OT_3DXP_XY", "OT_3DYP_XY", "OT_3DYP_YZ", "OT_3DZP_YZ", "OT_3DZP_ZX", "UNR_3DL"]
SITE = {n: i for i, n in enumerate(SITES)}

# Contraction modes of the reference build, pinned against the reference's
# own CUDA output on a B200 (tests/golden).  The CUDA kernels compile the same
# table (voxelizer_b200/csrc/vxb_sites.inc), which is parsed here so that the
# checker and the product always evaluate identical expression forms.
SITES_INC = os.path.join(os.path.dirname(HERE), "voxelizer_b200", "csrc", "vxb_sites.inc")


def _read_sites(path=SITES_INC):
    """{site: mode} for scalar sites, {site: [mode per node type]} for the
    sites whose mode depends on the node type."""
    out = {}
    with open(path) as fh:
        for line in fh:
            line = line.strip()
            if not line.startswith("constexpr int "):
                continue
            name, val = line[len("constexpr int "):].rstrip(";").split("=")
            name, val = name.strip(), val.strip()
            if name.endswith("]"):
                out[name[:name.index("[")]] = [int(x) for x in val.strip("{}").split(",")]
            else:
                out[name] = int(val)
    return out


PINNED_FMA = _read_sites()


def fma_sites(model=None, node_type=1):
    """64-entry site array for one node type from a {site name: mode or
    [mode per node type]} dict (None: pinned)."""
    arr = [0] * 64
    for k, v in (PINNED_FMA if model is None else model).items():
        arr[SITE[k]] = int(v[node_type] if isinstance(v, (list, tuple)) else v)
    return arr

NODE_BYTES = {0: 1, 1: 2, 2: 8, 3: 2, 4: 4}
PARTIAL_NODE = 2


class _Params(ctypes.Structure):
    _fields_ = [("node_type", ctypes.c_int), ("node_output", ctypes.c_int), ("materials", ctypes.c_int),
                ("by_cube_length", ctypes.c_int), ("max_dim", ctypes.c_uint32), ("cube_length", ctypes.c_double),
                ("vox_split", ctypes.c_uint32 * 3), ("mat_split", ctypes.c_uint32 * 3),
                ("fma_sites", ctypes.c_uint8 * 64), ("threads", ctypes.c_int), ("space", ctypes.c_int),
                ("part", ctypes.c_uint32 * 4), ("rotate_x", ctypes.c_int)]


class Info(ctypes.Structure):
    _fields_ = [("dims", ctypes.c_uint32 * 3), ("out_bytes", ctypes.c_uint64), ("voxel_length", ctypes.c_double),
                ("min_vertex", ctypes.c_double * 3), ("resolution", ctypes.c_uint32 * 3),
                ("x_splits", ctypes.c_uint32), ("n_conflicts", ctypes.c_uint64), ("n_surface", ctypes.c_uint64),
                ("prune_passes", ctypes.c_uint32)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run `make -C oracle oracle`")
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.orc_plan.restype = ctypes.c_int
        _lib.orc_plan.argtypes = [ctypes.POINTER(_Params), ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(Info)]
        _lib.orc_voxelize.restype = ctypes.c_int
        _lib.orc_voxelize.argtypes = [ctypes.POINTER(_Params), ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p,
                                      ctypes.c_uint32, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p,
                                      ctypes.c_uint64, ctypes.c_void_p, ctypes.POINTER(Info)]
        _lib.orc_voxelize_winners.restype = ctypes.c_int
        _lib.orc_voxelize_winners.argtypes = _lib.orc_voxelize.argtypes + [ctypes.c_void_p, ctypes.c_void_p]
    return _lib


def _params(node_type, nodes, materials, size, vox, mat, fma_model, threads, part=None, rotate_x=False):
    p = _Params()
    p.node_type = int(node_type)
    p.node_output = int(bool(nodes))
    p.materials = int(bool(materials))
    p.by_cube_length = int(isinstance(size, float))
    p.max_dim = 0 if isinstance(size, float) else int(size)
    p.cube_length = float(size) if isinstance(size, float) else 0.0
    p.vox_split[:] = list(vox)
    p.mat_split[:] = list(mat)
    p.fma_sites[:] = fma_sites(fma_model, int(node_type))
    p.threads = int(threads)
    if part is not None:   # device space: yz partition (y0, y1, z0, z1) of the grid
        p.space = 1
        p.part[:] = [int(v) for v in part]
    p.rotate_x = int(bool(rotate_x))
    return p


def out_dtype(node_type, nodes):
    if not nodes:
        return np.uint32
    return {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}[NODE_BYTES[node_type]]


def plan(mesh, node_type, nodes, size, vox=(1024, 512, 512), part=None, rotate_x=False):
    p = _params(node_type, nodes, 0, size, vox, (512, 512, 512), None, 0, part, rotate_x)
    info = Info()
    rc = lib().orc_plan(ctypes.byref(p), mesh.vertices.ctypes.data, mesh.n_vertices, ctypes.byref(info))
    if rc:
        raise RuntimeError(f"orc_plan failed: {rc}")
    return info


def voxelize(mesh, node_type, nodes, materials, size, vox=(1024, 512, 512), mat=(512, 512, 512),
             fma_model=None, threads=0, want_conflicts=False, part=None, rotate_x=False):
    """Returns (output array (flat), Info, conflict mask or None).  `part`
    (y0, y1, z0, z1) voxelizes that partition as a device space."""
    p = _params(node_type, nodes, materials, size, vox, mat, fma_model, threads, part, rotate_x)
    info = Info()
    L = lib()
    rc = L.orc_plan(ctypes.byref(p), mesh.vertices.ctypes.data, mesh.n_vertices, ctypes.byref(info))
    if rc:
        raise RuntimeError(f"orc_plan failed: {rc}")
    dt = out_dtype(node_type, nodes)
    out = np.empty(int(info.out_bytes) // np.dtype(dt).itemsize, dtype=dt)
    conf = np.zeros(out.size if nodes else 0, np.uint8) if want_conflicts else None
    mats = mesh.materials if mesh.materials is not None else np.zeros(mesh.n_triangles, np.uint8)
    rc = L.orc_voxelize(ctypes.byref(p), mesh.vertices.ctypes.data, mesh.n_vertices, mesh.indices.ctypes.data,
                        mesh.n_triangles, mats.ctypes.data, mesh.n_materials, out.ctypes.data, out.nbytes,
                        conf.ctypes.data if conf is not None else None, ctypes.byref(info))
    if rc:
        raise RuntimeError(f"orc_voxelize failed: {rc}")
    return out, info, conf


def voxelize_winners(mesh, size, vox=(1024, 512, 512), mat=(512, 512, 512), fma_model=None, threads=0):
    """PartialNode with materials: (output, Info, conflict mask, winning
    triangle per node (0xFFFFFFFF off the surface), winning class per node)."""
    p = _params(PARTIAL_NODE, 1, 1, size, vox, mat, fma_model, threads)
    info = Info()
    L = lib()
    rc = L.orc_plan(ctypes.byref(p), mesh.vertices.ctypes.data, mesh.n_vertices, ctypes.byref(info))
    if rc:
        raise RuntimeError(f"orc_plan failed: {rc}")
    out = np.empty(int(info.out_bytes) // 8, dtype=np.uint64)
    conf = np.zeros(out.size, np.uint8)
    tri = np.full(out.size, 0xFFFFFFFF, np.uint32)
    cls = np.zeros(out.size, np.uint8)
    mats = mesh.materials if mesh.materials is not None else np.zeros(mesh.n_triangles, np.uint8)
    rc = L.orc_voxelize_winners(ctypes.byref(p), mesh.vertices.ctypes.data, mesh.n_vertices, mesh.indices.ctypes.data,
                                mesh.n_triangles, mats.ctypes.data, mesh.n_materials, out.ctypes.data, out.nbytes,
                                conf.ctypes.data, ctypes.byref(info), tri.ctypes.data, cls.ctypes.data)
    if rc:
        raise RuntimeError(f"orc_voxelize_winners failed: {rc}")
    return out, info, conf, tri, cls


def surface_hits(mesh, node_type, size, grid=0, vox=(1024, 512, 512), mat=(512, 512, 512), fma_model=None):
    """Every surface hit of one lattice as an (n, 2) array of (triangle, node
    index) rows, evaluated with `fma_model` (None: the pinned modes)."""
    p = _params(node_type, 1, 1, size, vox, mat, fma_model, 0)
    L = lib()
    L.orc_surface_hits.restype = ctypes.c_longlong
    L.orc_surface_hits.argtypes = [ctypes.POINTER(_Params), ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p,
                                   ctypes.c_uint32, ctypes.c_int, ctypes.c_void_p, ctypes.c_uint64]
    cap = 1 << 16
    while True:
        buf = np.empty(cap, np.uint64)
        n = L.orc_surface_hits(ctypes.byref(p), mesh.vertices.ctypes.data, mesh.n_vertices, mesh.indices.ctypes.data,
                               mesh.n_triangles, int(grid), buf.ctypes.data, cap)
        if n < 0:
            raise RuntimeError(f"orc_surface_hits failed: {n}")
        if n <= cap:
            buf = buf[:n]
            return np.stack([(buf >> np.uint64(32)).astype(np.int64), (buf & np.uint64(0xFFFFFFFF)).astype(np.int64)], 1)
        cap = int(n)
