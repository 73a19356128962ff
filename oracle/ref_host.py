"""ctypes binding of oracle/_ref/libvoxhost.so: the reference's own public
API (vox::Voxelizer<Node> from its src/host_side.cpp and src/voxelizer.cu,
built by ``make -C oracle refhost``; see ref_host.cu).

TEST INFRASTRUCTURE ONLY: loaded by tests/ and by bench.py's reference arm.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libvoxhost.so")
NODE_DTYPE = {0: np.uint8, 1: np.uint16, 2: np.uint64, 3: np.uint16, 4: np.uint32}

_lib = None


def available():
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        L.refh_dims.restype = ctypes.c_int
        L.refh_dims.argtypes = [ctypes.c_int, vp, ctypes.c_uint32, vp, ctypes.c_uint32, ctypes.c_int, ctypes.c_uint32,
                                ctypes.c_double, ctypes.c_uint32, ctypes.c_int, vp]
        L.refh_voxelize.restype = ctypes.c_int
        L.refh_voxelize.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint32, ctypes.c_double, vp,
                                    vp, vp, ctypes.c_uint32, vp, ctypes.c_uint32, vp, ctypes.c_uint32, vp,
                                    ctypes.c_uint64, vp, ctypes.POINTER(ctypes.c_double)]
        L.refh_last_error.restype = ctypes.c_char_p
        _lib = L
    return _lib


def _size(size):
    return (1, 0, float(size)) if isinstance(size, float) else (0, int(size), 0.0)


def array_dimensions(mesh, node_type, size, max_x=1024, slice_x=False):
    """Voxelizer<Node>::getArrayDimensions (host code; no GPU needed)."""
    L = lib()
    by_cube, md, cube = _size(size)
    d = np.zeros(3, np.uint32)
    rc = L.refh_dims(int(node_type), mesh.vertices.ctypes.data, mesh.n_vertices, mesh.indices.ctypes.data,
                     mesh.n_triangles, by_cube, md, cube, int(max_x), int(bool(slice_x)), d.ctypes.data)
    if rc:
        raise RuntimeError(f"refh_dims failed ({rc}): {L.refh_last_error().decode()}")
    return tuple(int(x) for x in d)


def voxelize(mesh, node_type, nodes, size, vox=(1024, 512, 512), mat=(512, 512, 512), materials=True,
             out=None):
    """voxelizeToNodesToRAM (nodes=1) or voxelizeToRAM (nodes=0) through the
    reference's own API on the current GPU.  Returns (array, dims, ms)."""
    L = lib()
    by_cube, md, cube = _size(size)
    vs = np.array(vox, np.uint32)
    ms = np.array(mat, np.uint32)
    dims = np.zeros(3, np.uint32)
    t = ctypes.c_double(0.0)
    mats = mesh.materials if (materials and mesh.materials is not None) else None
    args = [int(node_type), int(nodes), by_cube, md, cube, vs.ctypes.data, ms.ctypes.data, mesh.vertices.ctypes.data,
            mesh.n_vertices, mesh.indices.ctypes.data, mesh.n_triangles,
            mats.ctypes.data if mats is not None else None, mesh.n_materials if mats is not None else 0]
    if out is None:
        rc = L.refh_voxelize(*args, None, 0, dims.ctypes.data, ctypes.byref(t))
        if rc:
            raise RuntimeError(f"refh_voxelize failed ({rc}): {L.refh_last_error().decode()}")
        n = int(dims[0]) * int(dims[1]) * int(dims[2])
        out = np.empty(n if nodes else n // 32, NODE_DTYPE[node_type] if nodes else np.uint32)
    rc = L.refh_voxelize(*args, out.ctypes.data, out.nbytes, dims.ctypes.data, ctypes.byref(t))
    if rc:
        raise RuntimeError(f"refh_voxelize failed ({rc}): {L.refh_last_error().decode()}")
    return out, tuple(int(x) for x in dims), t.value
