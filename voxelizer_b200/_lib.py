"""ctypes binding of libvxb.so (include/vxb.h).

The shared library is built in-tree (voxelizer_b200/libvxb.so, see
build.py).  There is no fallback: if the library is missing or fails to
load, every call raises.
"""

from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libvxb.so")

VXB_OK = 0
STATUS = {0: "VXB_OK", -1: "VXB_EINVAL", -2: "VXB_ENOMEM", -3: "VXB_ECUDA", -4: "VXB_EUNSUPPORTED",
          -5: "VXB_ETIMEDOUT", -6: "VXB_EOVERFLOW", -7: "VXB_ENOMATERIALS"}

SHORT, LONG, PARTIAL, SHORT_FCC, LONG_FCC = range(5)
NODE_BYTES = {SHORT: 1, LONG: 2, PARTIAL: 8, SHORT_FCC: 2, LONG_FCC: 4}

# Every extern "C" symbol include/vxb.h declares.
EXPORTS = ["vxb_last_error", "vxb_version", "vxb_create", "vxb_destroy", "vxb_set_materials",
           "vxb_set_material_output", "vxb_verbose_output", "vxb_plan", "vxb_get_array_dimensions",
           "vxb_voxelize_to_host", "vxb_voxelize_to_device", "vxb_last_launch_count", "vxb_set_profiling",
           "vxb_stage_times", "vxb_stage_timeline", "vxb_scan_counts", "vxb_voxelize_bits_noalloc", "vxb_trim_cache", "vxb_batch_create",
           "vxb_batch_destroy", "vxb_batch_add", "vxb_batch_clear", "vxb_batch_run", "vxb_batch_last_launch_count",
           "vxb_last_stats", "vxb_plan_parts", "vxb_voxelize_parts_to_device", "vxb_voxelize_parts_to_host",
           "vxb_plan_slice", "vxb_voxelize_slice_to_device", "vxb_voxelize_slice_to_host", "vxb_set_autotune",
           "vxb_autotune_state", "vxb_noalloc_status", "vxb_bounding_box"]

BATCH_GRAPH = 1


class VxbError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


class Uint3(ctypes.Structure):
    _fields_ = [("x", ctypes.c_uint32), ("y", ctypes.c_uint32), ("z", ctypes.c_uint32)]


class Request(ctypes.Structure):
    _fields_ = [("by_cube_length", ctypes.c_int), ("max_dimension", ctypes.c_uint32),
                ("cube_length", ctypes.c_double), ("vox_split_res", Uint3), ("mat_split_res", Uint3)]


class GridInfo(ctypes.Structure):
    _fields_ = [("dim", Uint3), ("bytes", ctypes.c_uint64), ("count", ctypes.c_uint64),
                ("voxel_length", ctypes.c_double), ("min_vertex", ctypes.c_double * 3),
                ("max_vertex", ctypes.c_double * 3), ("resolution", Uint3), ("x_splits", ctypes.c_uint32),
                ("location", Uint3), ("partition", ctypes.c_uint32 * 4)]

    @property
    def dims(self):
        return (int(self.dim.x), int(self.dim.y), int(self.dim.z))


class Stats(ctypes.Structure):
    _fields_ = [("units", ctypes.c_uint32), ("work_triangles", ctypes.c_uint32),
                ("solid_candidates", ctypes.c_uint32), ("surface_columns", ctypes.c_uint32),
                ("surface_hits", ctypes.c_uint32), ("surface_voxels", ctypes.c_uint32),
                ("surface_triangles", ctypes.c_uint32 * 3), ("grid_words", ctypes.c_uint64)]

    def as_dict(self):
        return {k: (list(getattr(self, k)) if k == "surface_triangles" else int(getattr(self, k)))
                for k, _ in self._fields_}


_lib = None


def lib():
    """Loads libvxb.so once; raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m voxelizer_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    P = ctypes.POINTER
    vp = ctypes.c_void_p
    sig = {
        "vxb_last_error": (ctypes.c_char_p, []),
        "vxb_version": (ctypes.c_char_p, []),
        "vxb_create": (ctypes.c_int, [P(vp), ctypes.c_int, vp, vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int]),
        "vxb_destroy": (ctypes.c_int, [vp]),
        "vxb_trim_cache": (ctypes.c_int, []),
        "vxb_batch_create": (ctypes.c_int, [P(vp), ctypes.c_int]),
        "vxb_batch_destroy": (ctypes.c_int, [vp]),
        "vxb_batch_add": (ctypes.c_int, [vp, vp, ctypes.c_int, P(Request), vp, ctypes.c_uint64, P(GridInfo)]),
        "vxb_batch_clear": (ctypes.c_int, [vp]),
        "vxb_batch_run": (ctypes.c_int, [vp, vp, ctypes.c_int]),
        "vxb_batch_last_launch_count": (ctypes.c_int, [vp, P(ctypes.c_uint32)]),
        "vxb_last_stats": (ctypes.c_int, [vp, P(Stats)]),
        "vxb_set_materials": (ctypes.c_int, [vp, vp, ctypes.c_uint32]),
        "vxb_set_material_output": (ctypes.c_int, [vp, ctypes.c_int]),
        "vxb_verbose_output": (ctypes.c_int, [vp, ctypes.c_int]),
        "vxb_plan": (ctypes.c_int, [vp, ctypes.c_int, P(Request), P(GridInfo)]),
        "vxb_get_array_dimensions": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_uint32, ctypes.c_double,
                                                    ctypes.c_uint32, ctypes.c_int, P(Uint3)]),
        "vxb_voxelize_to_host": (ctypes.c_int, [vp, ctypes.c_int, P(Request), vp, ctypes.c_uint64, P(GridInfo)]),
        "vxb_voxelize_to_device": (ctypes.c_int, [vp, ctypes.c_int, P(Request), vp, ctypes.c_uint64, vp,
                                                  P(GridInfo)]),
        "vxb_last_launch_count": (ctypes.c_int, [vp, P(ctypes.c_uint32)]),
        "vxb_set_profiling": (ctypes.c_int, [vp, ctypes.c_int]),
        "vxb_stage_times": (ctypes.c_int, [vp, P(ctypes.c_float), ctypes.c_uint32]),
        "vxb_stage_timeline": (ctypes.c_int, [vp, P(ctypes.c_float), ctypes.c_uint32]),
        "vxb_scan_counts": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, P(ctypes.c_uint32),
                                           P(ctypes.c_uint32), ctypes.c_void_p]),
        "vxb_plan_parts": (ctypes.c_int, [vp, ctypes.c_int, P(Request), ctypes.c_uint32, ctypes.c_uint32,
                                          P(GridInfo)]),
        "vxb_voxelize_parts_to_device": (ctypes.c_int, [vp, ctypes.c_int, P(Request), ctypes.c_uint32,
                                                        ctypes.c_uint32, P(vp), P(ctypes.c_uint64), vp,
                                                        P(GridInfo)]),
        "vxb_voxelize_parts_to_host": (ctypes.c_int, [vp, ctypes.c_int, P(Request), ctypes.c_uint32,
                                                      ctypes.c_uint32, P(vp), P(ctypes.c_uint64), P(GridInfo)]),
        "vxb_set_autotune": (ctypes.c_int, [ctypes.c_int, ctypes.c_char_p]),
        "vxb_autotune_state": (ctypes.c_int, [P(ctypes.c_uint32), ctypes.c_char_p, ctypes.c_uint64]),
        "vxb_plan_slice": (ctypes.c_int, [vp, P(Request), ctypes.c_int, ctypes.c_uint32, P(GridInfo)]),
        "vxb_voxelize_slice_to_device": (ctypes.c_int, [vp, P(Request), ctypes.c_int, ctypes.c_uint32, vp,
                                                        ctypes.c_uint64, vp, P(GridInfo)]),
        "vxb_voxelize_slice_to_host": (ctypes.c_int, [vp, P(Request), ctypes.c_int, ctypes.c_uint32, vp,
                                                      ctypes.c_uint64, P(GridInfo)]),
        "vxb_voxelize_bits_noalloc": (ctypes.c_int, [vp, vp, ctypes.c_uint32, ctypes.c_uint32, P(ctypes.c_double),
                                                     P(ctypes.c_double), P(Request), vp, ctypes.c_uint64, vp,
                                                     P(GridInfo)]),
        "vxb_noalloc_status": (ctypes.c_int, []),
        "vxb_bounding_box": (ctypes.c_int, [vp, P(ctypes.c_double), P(ctypes.c_double)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def check(status):
    if status != VXB_OK:
        msg = lib().vxb_last_error()
        raise VxbError(status, msg.decode() if msg else "")
    return status


def make_request(size, vox_split=(1024, 512, 512), mat_split=(512, 512, 512)):
    """``size``: int -> maxDimension, float -> cubeLength (the two overloads
    of every Voxelizer::voxelize* member)."""
    r = Request()
    if isinstance(size, float):
        r.by_cube_length, r.max_dimension, r.cube_length = 1, 0, float(size)
    else:
        r.by_cube_length, r.max_dimension, r.cube_length = 0, int(size), 0.0
    r.vox_split_res = Uint3(*[int(v) for v in vox_split])
    r.mat_split_res = Uint3(*[int(v) for v in mat_split])
    return r


def set_autotune(mode, cache_path=None):
    """vxb_set_autotune: 0 default launch shapes, 1 tune online, 2 use the
    cache file's shapes."""
    check(lib().vxb_set_autotune(int(mode), cache_path.encode() if cache_path else None))


def autotune_state():
    """(settled buckets, JSON text of their shapes)."""
    n = ctypes.c_uint32()
    buf = ctypes.create_string_buffer(1 << 16)
    check(lib().vxb_autotune_state(ctypes.byref(n), buf, len(buf)))
    return int(n.value), buf.value.decode()
