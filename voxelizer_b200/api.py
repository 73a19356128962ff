"""Python mirror of the reference's ``vox::Voxelizer<Node>`` interface
(include/voxelizer.h), over the C ABI of libvxb.so.

Member names, argument meaning and defaults follow the reference:
``voxelizeToRAM`` returns the plain solid bit array, ``voxelizeToNodesToRAM``
the node grid; an ``int`` size is a maxDimension, a ``float`` size a
cubeLength.  Results are numpy arrays with the reference's byte layout
(``uint32`` words for bit arrays; ``uint8`` / ``uint16`` / ``uint64`` /
``uint16`` / ``uint32`` per node for ShortNode / LongNode / PartialNode /
ShortFCCNode / LongFCCNode).  Device variants write into a caller-owned
device buffer (any object with ``data_ptr()``, e.g. a torch CUDA tensor).
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import LONG, LONG_FCC, NODE_BYTES, PARTIAL, SHORT, SHORT_FCC, VxbError, check, lib, make_request  # noqa: F401

NODE_DTYPE = {SHORT: np.uint8, LONG: np.uint16, PARTIAL: np.uint64, SHORT_FCC: np.uint16, LONG_FCC: np.uint32}
DEFAULT_VOX = (1024, 512, 512)
DEFAULT_MAT = (512, 512, 512)


class Voxelizer:
    """One mesh, one node type (the template argument of the reference)."""

    def __init__(self, vertices, indices, materials=None, n_unique_materials=None, node_type=SHORT, device=0):
        v = np.ascontiguousarray(vertices, dtype=np.float32).reshape(-1)
        i = np.ascontiguousarray(indices, dtype=np.uint32).reshape(-1)
        if v.size % 3 or i.size % 3:
            raise ValueError("vertices and indices must hold 3 values per vertex / triangle")
        self.node_type = int(node_type)
        self.n_vertices = v.size // 3
        self.n_triangles = i.size // 3
        h = ctypes.c_void_p()
        check(lib().vxb_create(ctypes.byref(h), self.node_type, v.ctypes.data, i.ctypes.data, self.n_vertices,
                               self.n_triangles, int(device)))
        self._h = h
        if materials is not None:
            self.setMaterials(materials, n_unique_materials)

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().vxb_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- configuration (include/voxelizer.h:862-866) --
    def setMaterials(self, materials, n_unique_materials):
        m = np.ascontiguousarray(materials, dtype=np.uint8).reshape(-1)
        if m.size != self.n_triangles:
            raise ValueError("one material per triangle is required")
        if n_unique_materials is None:
            n_unique_materials = int(m.max()) + 1 if m.size else 0
        check(lib().vxb_set_materials(self._h, m.ctypes.data, int(n_unique_materials)))

    def setMaterialOutput(self, enable):
        check(lib().vxb_set_material_output(self._h, int(bool(enable))))

    def verboseOutput(self, enable):
        check(lib().vxb_verbose_output(self._h, int(bool(enable))))

    # -- planning --
    def plan(self, nodes, size, voxSplitRes=DEFAULT_VOX, matSplitRes=DEFAULT_MAT):
        info = _lib.GridInfo()
        r = make_request(size, voxSplitRes, matSplitRes)
        check(lib().vxb_plan(self._h, int(bool(nodes)), ctypes.byref(r), ctypes.byref(info)))
        return info

    def getArrayDimensions(self, size, maxInternalXSize=1024, sliceAlongX=False):
        d = _lib.Uint3()
        cube = isinstance(size, float)
        check(lib().vxb_get_array_dimensions(self._h, int(cube), 0 if cube else int(size), float(size) if cube else 0.0,
                                             int(maxInternalXSize), int(bool(sliceAlongX)), ctypes.byref(d)))
        return (int(d.x), int(d.y), int(d.z))

    # -- voxelization to host memory --
    def _to_host(self, nodes, size, voxSplitRes, matSplitRes, out=None):
        info = self.plan(nodes, size, voxSplitRes, matSplitRes)
        dt = NODE_DTYPE[self.node_type] if nodes else np.uint32
        if out is None:
            out = np.empty(int(info.count), dtype=dt)
        elif out.nbytes < info.bytes:
            raise ValueError("output buffer too small")
        r = make_request(size, voxSplitRes, matSplitRes)
        check(lib().vxb_voxelize_to_host(self._h, int(bool(nodes)), ctypes.byref(r), out.ctypes.data, out.nbytes,
                                         ctypes.byref(info)))
        return out, info

    def voxelizeToRAM(self, size=256, voxSplitRes=DEFAULT_VOX, out=None):
        """Plain solid voxelization: uint32 words, shape info.dims (voxels)."""
        return self._to_host(0, size, voxSplitRes, DEFAULT_MAT, out)

    def voxelizeToNodesToRAM(self, size=256, voxSplitRes=DEFAULT_VOX, matSplitRes=DEFAULT_MAT, out=None):
        """Node grid with boundary ids (and materials when enabled)."""
        return self._to_host(1, size, voxSplitRes, matSplitRes, out)

    # -- voxelization into a caller-owned device buffer --
    def voxelize_device(self, nodes, size, out, voxSplitRes=DEFAULT_VOX, matSplitRes=DEFAULT_MAT, stream=None):
        """``out`` exposes data_ptr() and nbytes (torch tensor); ``stream``
        is a raw cudaStream_t handle (int) or None for the default stream.
        Returns the GridInfo; the work is enqueued on ``stream``."""
        info = _lib.GridInfo()
        r = make_request(size, voxSplitRes, matSplitRes)
        nbytes = out.numel() * out.element_size() if hasattr(out, "element_size") else int(out.nbytes)
        check(lib().vxb_voxelize_to_device(self._h, int(bool(nodes)), ctypes.byref(r), ctypes.c_void_p(out.data_ptr()),
                                           nbytes, ctypes.c_void_p(stream or 0), ctypes.byref(info)))
        return info

    # -- slices (voxelizeSlice / voxelizeSliceToRAM, include/voxelizer.h:765-795) --
    @staticmethod
    def _slice_request(size, voxSplitRes, matSplitRes):
        # The reference's slice members take uint2 split sizes (a, b) and use
        # (a, b, b) (src/host_side.cpp:1966-1972).
        vs = tuple(voxSplitRes) if len(voxSplitRes) == 3 else (voxSplitRes[0], voxSplitRes[1], voxSplitRes[1])
        ms = tuple(matSplitRes) if len(matSplitRes) == 3 else (matSplitRes[0], matSplitRes[1], matSplitRes[1])
        return make_request(size, vs, ms)

    def planSlice(self, size, direction, slice, voxSplitRes=(1024, 512), matSplitRes=(512, 512)):
        info = _lib.GridInfo()
        r = self._slice_request(size, voxSplitRes, matSplitRes)
        check(lib().vxb_plan_slice(self._h, ctypes.byref(r), int(direction), int(slice), ctypes.byref(info)))
        return info

    def voxelizeSliceToRAM(self, size, direction, slice, voxSplitRes=(1024, 512), matSplitRes=(512, 512), out=None):
        """Node array of slice ``slice`` (1 .. resolution, counting the
        padding row as 0) along ``direction`` (1: y, 2: z): three layers along
        that axis, the middle one the slice.  Returns (array, GridInfo)."""
        info = self.planSlice(size, direction, slice, voxSplitRes, matSplitRes)
        if out is None:
            out = np.empty(int(info.count), dtype=NODE_DTYPE[self.node_type])
        elif out.nbytes < info.bytes:
            raise ValueError("output buffer too small")
        r = self._slice_request(size, voxSplitRes, matSplitRes)
        check(lib().vxb_voxelize_slice_to_host(self._h, ctypes.byref(r), int(direction), int(slice),
                                               out.ctypes.data, out.nbytes, ctypes.byref(info)))
        return out, info

    def voxelize_slice_device(self, size, direction, slice, out, voxSplitRes=(1024, 512), matSplitRes=(512, 512),
                              stream=None):
        info = _lib.GridInfo()
        r = self._slice_request(size, voxSplitRes, matSplitRes)
        nbytes = out.numel() * out.element_size() if hasattr(out, "element_size") else int(out.nbytes)
        check(lib().vxb_voxelize_slice_to_device(self._h, ctypes.byref(r), int(direction), int(slice),
                                                 ctypes.c_void_p(out.data_ptr()), nbytes,
                                                 ctypes.c_void_p(stream or 0), ctypes.byref(info)))
        return info

    # -- devConfig partitions (voxelize(..., devConfig, ...), include/voxelizer.h:718-770) --
    def planParts(self, nodes, size, devConfig, voxSplitRes=DEFAULT_VOX, matSplitRes=DEFAULT_MAT):
        dy, dz = (int(v) for v in devConfig)
        infos = (_lib.GridInfo * (dy * dz))()
        r = make_request(size, voxSplitRes, matSplitRes)
        check(lib().vxb_plan_parts(self._h, int(bool(nodes)), ctypes.byref(r), dy, dz, infos))
        return list(infos)

    def voxelizePartsToRAM(self, nodes, size, devConfig, voxSplitRes=DEFAULT_VOX, matSplitRes=DEFAULT_MAT):
        """One result per partition of the yz voxel range (devConfig (dev_y,
        dev_z), y fastest), each voxelized as the reference's devices do.
        Returns a list of (array, GridInfo); GridInfo.location is the
        partition's (0, y, z)."""
        dy, dz = (int(v) for v in devConfig)
        infos = self.planParts(nodes, size, devConfig, voxSplitRes, matSplitRes)
        dt = NODE_DTYPE[self.node_type] if nodes else np.uint32
        outs = [np.empty(int(i.count), dtype=dt) for i in infos]
        ptrs = (ctypes.c_void_p * len(outs))(*[o.ctypes.data for o in outs])
        sizes = (ctypes.c_uint64 * len(outs))(*[o.nbytes for o in outs])
        arr = (_lib.GridInfo * len(outs))()
        r = make_request(size, voxSplitRes, matSplitRes)
        check(lib().vxb_voxelize_parts_to_host(self._h, int(bool(nodes)), ctypes.byref(r), dy, dz, ptrs, sizes, arr))
        return list(zip(outs, list(arr)))

    def set_profiling(self, enable, serial=False):
        """Stage events on (off with enable False); serial runs the stages
        one after another so that each stage's time is its own."""
        check(lib().vxb_set_profiling(self._h, (2 if serial else 1) if enable else 0))

    STAGES = ("solid", "surface", "prune", "emit", "merge", "surface_work")

    def stage_times(self):
        """Milliseconds per stage of the last call (-1: stage did not run)."""
        buf = (ctypes.c_float * len(self.STAGES))()
        check(lib().vxb_stage_times(self._h, buf, len(self.STAGES)))
        return dict(zip(self.STAGES, [float(x) for x in buf]))

    def stage_timeline(self):
        """(start, end) in ms after the solid stage's start, per stage of the
        last call (NaN: stage did not run)."""
        buf = (ctypes.c_float * (2 * len(self.STAGES)))()
        check(lib().vxb_stage_timeline(self._h, buf, len(self.STAGES)))
        return {k: (float(buf[2 * i]), float(buf[2 * i + 1])) for i, k in enumerate(self.STAGES)}

    def last_launch_count(self):
        n = ctypes.c_uint32()
        check(lib().vxb_last_launch_count(self._h, ctypes.byref(n)))
        return int(n.value)

    def last_stats(self):
        """Work counters of the last call (vxb_last_stats)."""
        st = _lib.Stats()
        check(lib().vxb_last_stats(self._h, ctypes.byref(st)))
        return st.as_dict()


class VoxelizerBatch:
    """Several voxelizers' meshes run through one sequence of launches
    (vxb_batch_*).  Every mesh gets its own request and device output;
    results equal the single-mesh calls.  ``graph=True`` captures the
    launches once and replays them on later runs of the same batch."""

    def __init__(self, device=0):
        h = ctypes.c_void_p()
        check(lib().vxb_batch_create(ctypes.byref(h), int(device)))
        self._h = h
        self._keep = []

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().vxb_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def add(self, voxelizer, nodes, size, out, voxSplitRes=DEFAULT_VOX, matSplitRes=DEFAULT_MAT):
        """Adds one mesh; ``out`` exposes data_ptr() (a device tensor)."""
        info = _lib.GridInfo()
        r = make_request(size, voxSplitRes, matSplitRes)
        nbytes = out.numel() * out.element_size() if hasattr(out, "element_size") else int(out.nbytes)
        check(lib().vxb_batch_add(self._h, voxelizer._h, int(bool(nodes)), ctypes.byref(r),
                                  ctypes.c_void_p(out.data_ptr()), nbytes, ctypes.byref(info)))
        self._keep.append((voxelizer, out))
        return info

    def clear(self):
        check(lib().vxb_batch_clear(self._h))
        self._keep = []

    def run(self, stream=None, graph=False):
        check(lib().vxb_batch_run(self._h, ctypes.c_void_p(stream or 0), _lib.BATCH_GRAPH if graph else 0))

    def last_launch_count(self):
        n = ctypes.c_uint32()
        check(lib().vxb_batch_last_launch_count(self._h, ctypes.byref(n)))
        return int(n.value)
