"""vxb_voxelize_bits_noalloc against vxb_voxelize_to_device.

vxb_voxelize_bits_noalloc serves callers that cannot allocate device memory:
solvers that reserve the whole GPU for their own memory pool before they
voxelize, or that cannot afford the device-wide synchronization of
cudaMalloc / cudaFree in the middle of a time step.  Its work lists live in a
fixed array inside the library that every call reuses, so the GPU check runs
two different requests back to back on that array and compares each result
bit for bit with the allocating entry point's.  Errors that only the GPU sees (an
index past the vertex buffer) are read back with vxb_noalloc_status once
the call's stream has finished.  This file is named to be collected last.
"""

import ctypes

import numpy as np
import pytest

from voxelizer_b200 import _lib, scenes
from voxelizer_b200.api import LONG, Voxelizer

MAX_TRIANGLES = 1 << 20


class _FakeBuffer:
    """Stands in for an output buffer in calls refused before any device work."""

    def data_ptr(self):
        return 256

    def numel(self):
        return 1

    def element_size(self):
        return 4


def _noalloc(lib, dv, di, n_v, n_t, mn, mx, req, out, stream=0):
    info = _lib.GridInfo()
    lo = (ctypes.c_double * 3)(*mn)
    hi = (ctypes.c_double * 3)(*mx)
    st = lib.vxb_voxelize_bits_noalloc(ctypes.c_void_p(dv), ctypes.c_void_p(di), n_v, n_t, lo, hi, ctypes.byref(req),
                                       ctypes.c_void_p(out.data_ptr()), out.numel() * out.element_size(),
                                       ctypes.c_void_p(stream), ctypes.byref(info))
    return st, info


def test_noalloc_rejects_oversized_requests():
    """Sizes beyond the fixed array are refused with a message naming the limit."""
    lib = _lib.lib()
    box = ((0.0, 0.0, 0.0), (1.0, 1.0, 1.0))
    st, _ = _noalloc(lib, 256, 256, 3, MAX_TRIANGLES + 1, *box, _lib.make_request(64), _FakeBuffer())
    assert st == -1
    assert b"1048576" in lib.vxb_last_error()
    # One yz subspace per voxel row and column: 200 x 200 subspaces.
    st, _ = _noalloc(lib, 256, 256, 3, 1, *box, _lib.make_request(200, vox_split=(1024, 1, 1)), _FakeBuffer())
    assert st == -1
    assert b"1024" in lib.vxb_last_error() and b"subspaces" in lib.vxb_last_error()
    # The candidate bound: 1M triangles over a 4096 x 4096 yz plane in 8 x 8
    # subspaces could list more than 2^32 (triangle, tile) candidates.
    slab = ((0.0, 0.0, 0.0), (0.01, 1.0, 1.0))
    st, _ = _noalloc(lib, 256, 256, 3, MAX_TRIANGLES, *slab, _lib.make_request(4096, vox_split=(1024, 512, 512)),
                     _FakeBuffer())
    assert st == -1
    assert b"2^32" in lib.vxb_last_error()
    # A voxel length so small that the resolution would wrap 32 bits.
    st, _ = _noalloc(lib, 256, 256, 3, 1, *box, _lib.make_request(1e-12), _FakeBuffer())
    assert st == -1


def _sphere_on_device(torch):
    v, i = scenes.icosphere(3, radius=1.0, center=(0.1, -0.2, 0.05))
    v = v.astype(np.float32)
    i = i.astype(np.uint32)
    return v, i, torch.from_numpy(v.reshape(-1)).cuda(), torch.from_numpy(i.reshape(-1).view(np.int32)).cuda()


@pytest.mark.gpu
def test_noalloc_reports_index_out_of_range():
    """An index >= n_vertices is caught on the device: the call reads vertex
    0 in its place (nothing past the vertex buffer), and the status call
    reports VXB_EINVAL once the stream has finished; the next valid call
    clears it."""
    torch = pytest.importorskip("torch")
    lib = _lib.lib()
    v, i, dv, di = _sphere_on_device(torch)
    with Voxelizer(v, i, node_type=LONG) as vx:
        info = vx.plan(0, 64)
    out = torch.zeros(int(info.count), dtype=torch.int32, device="cuda")
    bad = di.clone()
    bad[7] = v.shape[0] + 5
    st, _ = _noalloc(lib, dv.data_ptr(), bad.data_ptr(), v.shape[0], i.shape[0], info.min_vertex, info.max_vertex,
                     _lib.make_request(64), out)
    assert st == 0, lib.vxb_last_error()
    torch.cuda.synchronize()
    assert lib.vxb_noalloc_status() == -1
    assert b"index" in lib.vxb_last_error()
    st, _ = _noalloc(lib, dv.data_ptr(), di.data_ptr(), v.shape[0], i.shape[0], info.min_vertex, info.max_vertex,
                     _lib.make_request(64), out)
    assert st == 0
    torch.cuda.synchronize()
    assert lib.vxb_noalloc_status() == 0


@pytest.mark.gpu
def test_noalloc_on_a_non_default_stream():
    """Stream-ordered on the caller's stream: the result equals the
    allocating entry point's, and the status reads back clean."""
    torch = pytest.importorskip("torch")
    lib = _lib.lib()
    v, i, dv, di = _sphere_on_device(torch)
    with Voxelizer(v, i, node_type=LONG) as vx:
        info = vx.plan(0, 96)
        ref = torch.empty(int(info.count), dtype=torch.int32, device="cuda")
        vx.voxelize_device(0, 96, ref)
    torch.cuda.synchronize()
    s = torch.cuda.Stream()
    out = torch.full((int(info.count),), -1, dtype=torch.int32, device="cuda")
    with torch.cuda.stream(s):
        st, _ = _noalloc(lib, dv.data_ptr(), di.data_ptr(), v.shape[0], i.shape[0], info.min_vertex,
                         info.max_vertex, _lib.make_request(96), out, stream=s.cuda_stream)
    assert st == 0, lib.vxb_last_error()
    s.synchronize()
    assert lib.vxb_noalloc_status() == 0
    assert torch.equal(out, ref)


@pytest.mark.gpu
def test_noalloc_matches_device_entry_on_two_calls():
    torch = pytest.importorskip("torch")
    lib = _lib.lib()
    sv, si = scenes.icosphere(4, radius=1.0, center=(0.1, -0.2, 0.05))
    tv, ti = scenes.torus(96, 48, major=1.3, minor=0.35, center=(0.4, 0.3, -0.1))
    v = np.concatenate([sv, tv]).astype(np.float32)
    i = np.concatenate([si, ti + sv.shape[0]]).astype(np.uint32)
    dv = torch.from_numpy(v.reshape(-1)).cuda()
    di = torch.from_numpy(i.reshape(-1).view(np.int32)).cuda()
    # The second call reuses what the first one left in the array: a longer
    # triangle scan and another subspace table.  It voxelizes the sphere
    # alone (the leading triangles and vertices of the same device buffers).
    calls = [
        (v, i, 300, (1024, 64, 64)),
        (sv, si, 0.02, (256, 512, 512)),
    ]
    for verts, idx, size, vox in calls:
        with Voxelizer(verts, idx, node_type=LONG) as vx:
            ref_info = vx.plan(0, size, vox)
            ref = torch.empty(int(ref_info.count), dtype=torch.int32, device="cuda")
            vx.voxelize_device(0, size, ref, vox)
            out = torch.full((int(ref_info.count) + 7,), -1, dtype=torch.int32, device="cuda")
            st, info = _noalloc(lib, dv.data_ptr(), di.data_ptr(), verts.shape[0], idx.shape[0], ref_info.min_vertex,
                                ref_info.max_vertex, _lib.make_request(size, vox), out)
            assert st == 0, lib.vxb_last_error()
            torch.cuda.synchronize()
            assert info.dims == ref_info.dims
            assert info.bytes == ref_info.bytes and info.count == ref_info.count
            assert info.voxel_length == ref_info.voxel_length and info.x_splits == ref_info.x_splits
            assert int(ref.ne(0).sum()) > 0
            assert torch.equal(out[: ref.numel()], ref), f"bit array differs for request {size!r}"
            assert bool((out[ref.numel():] == -1).all()), "wrote past the result"
            assert lib.vxb_noalloc_status() == 0
