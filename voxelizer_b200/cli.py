"""Command-line voxelizer mirroring the reference's tester
(tests/src/main.cpp:197-450, initTests 1520-1580).

    python -m voxelizer_b200.cli MODEL.(obj|stl|ply|vtk) -r 256 [-x] [-m] [-L|-P|-F] \
        [-S DIR N | -A DIR | -D DY DZ] [-V X Y (Z)] [-M X Y (Z)] [-v] [-o OUT.npy]

Options keep the tester's letters and meaning: ``-r`` voxels along the
longest side, ``-d`` distance between voxel centres, ``-x`` plain voxel
output instead of nodes, ``-m`` materials with the tester's mapping
(triangle i gets material 1 + i % 7, eight unique materials, material
output on), ``-L`` / ``-P`` / ``-F`` the node type (``-L -F`` is the long FCC
node), ``-S DIR N`` slice N along direction DIR (voxelizeSliceToRAM, three
layers), ``-A DIR`` every slice along DIR placed into the full array as the
tester's applySlice does (1350-1434), ``-D DY DZ`` the simulated multi-device
partitions stitched as the tester's stitchNodeArrays does (1227-1262,
fetchResolution 1296-1311), ``-V`` / ``-M`` the internal voxel / material
split resolutions (two values with ``-S``, three otherwise), ``-v``
verbose, ``-u`` accepted (it only changes the tester's rendering).  The
tester renders the result with VTK; here the result is written as a numpy
array (``-o``) and summarised on stdout.
"""

from __future__ import annotations

import argparse
import sys
import time

import numpy as np

from . import api
from .meshio import MeshFormatError, load_mesh


def _node_type(a):
    if a.long:
        return api.LONG_FCC if a.fcc else api.LONG
    if a.fcc:
        return api.SHORT_FCC
    if a.part:
        return api.PARTIAL
    return api.SHORT


_NODE_NAMES = {api.SHORT: "ShortNode", api.LONG: "LongNode", api.PARTIAL: "PartialNode",
               api.SHORT_FCC: "ShortFCCNode", api.LONG_FCC: "LongFCCNode"}


def parser():
    p = argparse.ArgumentParser(prog="python -m voxelizer_b200.cli", description=__doc__.split("\n\n")[0])
    p.add_argument("filename", help="File to be voxelized (.obj, .stl, .ply, .vtk).")
    p.add_argument("-r", "--resolution", type=int, help="Number of voxels along longest side.")
    p.add_argument("-d", "--distance", type=float, help="Distance between voxel centers.")
    p.add_argument("-x", "--voxels", action="store_true", help="Produce voxel output instead of nodes.")
    p.add_argument("-m", "--materials", action="store_true", help="Produce materials output with a simple mapping.")
    p.add_argument("-L", "--long", action="store_true", help="Use the larger LongNode type.")
    p.add_argument("-P", "--part", action="store_true", help="Use the PartialNode type.")
    p.add_argument("-F", "--fcc", action="store_true", help="Use one of the FCC node types.")
    p.add_argument("-S", "--slice", type=int, nargs="+", metavar="N",
                   help="Produce a slice of the total voxelization (direction, slice number).")
    p.add_argument("-A", "--allSlice", type=int, metavar="DIR", help="Voxelizes and concatenates all slices.")
    p.add_argument("-D", "--multiDevice", type=int, nargs="+", metavar="N",
                   help="Simulate multiple devices and combine the results.")
    p.add_argument("-V", "--voxRes", type=int, nargs="+", metavar="N", help="Internal voxelization dimensions.")
    p.add_argument("-M", "--matRes", type=int, nargs="+", metavar="N",
                   help="Internal material voxelization dimensions.")
    p.add_argument("-v", "--verbose", action="store_true", help="Prints detailed information about the voxelization.")
    p.add_argument("-u", "--surface", action="store_true", help="Only renders the surface of the voxelization.")
    p.add_argument("-o", "--output", help="Write the result array to this .npy file.")
    p.add_argument("--device", type=int, default=0, help="CUDA device.")
    return p


_BID = {api.SHORT: (0x1F, 5, 0x7), api.LONG: (0xFF, 8, 0xFF), api.PARTIAL: (0xFF, 8, 0xFF),
        api.SHORT_FCC: (0xFFF, 12, 0xF), api.LONG_FCC: (0xFFFF, 16, 0xFF)}


def summarize(result, dims, nodes, node_type):
    """Text lines: grid size, solid count, boundary-id and material histograms."""
    X, Y, Z = dims
    lines = [f"dimensions: {X} x {Y} x {Z}"]
    if not nodes:
        lines.append(f"solid voxels: {int(np.unpackbits(result.view(np.uint8)).sum())}")
        return lines
    bmask, mshift, mmask = _BID[node_type]
    r = result.astype(np.uint64)
    bid = r & np.uint64(bmask)
    mat = (r >> np.uint64(mshift)) & np.uint64(mmask)
    lines.append(f"solid nodes: {int(np.count_nonzero(bid))} of {r.size}")
    ids, counts = np.unique(bid[bid != 0], return_counts=True)
    lines.append("boundary ids: " + ", ".join(f"{int(i)}:{int(c)}" for i, c in zip(ids, counts)))
    if np.any(mat):
        ms, mc = np.unique(mat[mat != 0], return_counts=True)
        lines.append("materials: " + ", ".join(f"{int(i)}:{int(c)}" for i, c in zip(ms, mc)))
    return lines


def check_args(a):
    """The tester's argument checks (tests/src/main.cpp:269-356); a message,
    or None when the arguments are usable."""
    if a.resolution is None and a.distance is None:
        return "No resolution or distance was given."
    for name in ("voxRes", "matRes"):
        v = getattr(a, name)
        if v is None:
            continue
        if a.slice is not None and len(v) != 2:
            return f"--{name} requires 2 arguments with --slice."
        if a.slice is None and len(v) != 3:
            return f"--{name} requires 3 arguments."
    if a.slice is not None:
        if len(a.slice) != 2:
            return "--slice requires 2 arguments."
        if a.slice[0] > 2 or a.slice[0] < 0:
            return "The direction of slice is > 2."
    if a.allSlice is not None and not 0 <= a.allSlice <= 2:
        return "The direction has to be between 0 and 2."
    if a.multiDevice is not None and len(a.multiDevice) != 2:
        return "--multiDevice: Device configuration needs two values."
    return None


def apply_slice(sl, k, nodes, res, direction):
    """applySlice for Cartesian nodes (tests/src/main.cpp:1396-1434): the
    middle layer of slice array ``sl`` becomes layer ``k`` of ``nodes``
    (x fastest, dimensions ``res``)."""
    X, Y, Z = res
    full = nodes.reshape(Z, Y, X)
    if direction == 0:
        full[:, :, k] = sl.reshape(Z, Y, 3)[:, :, 1]
    elif direction == 1:
        full[:, k, :] = sl.reshape(Z, 3, X)[:, 1, :]
    else:
        full[k] = sl.reshape(3, Y, X)[1]


def stitch(parts, dev_y, dev_z):
    """stitchNodeArrays with fetchResolution (tests/src/main.cpp:1227-1311):
    the inner nodes of every partition go to (1 + x, 1 + loc.y (dim.y - 2) + y,
    1 + loc.z (dim.z - 2) + z) of an array whose y / z extents are the summed
    partition extents without their padding plus 2.  The tester shifts x by
    one and assumes equal partition extents; both are kept, and nodes that
    land outside the array (the tester writes past its end there) are left
    out.  Returns (array, (X, Y, Z))."""
    if len(parts) == 1:
        arr, info = parts[0]
        return arr, info.dims
    X = parts[0][1].dims[0]
    Y = sum(i.dims[1] - 2 for _, i in parts) // dev_z + 2
    Z = sum(i.dims[2] - 2 for _, i in parts) // dev_y + 2
    out = np.zeros(X * Y * Z, dtype=parts[0][0].dtype)
    full = out.reshape(Z, Y, X)
    for arr, info in parts:
        sx, sy, sz = info.dims
        src = arr.reshape(sz, sy, sx)[1:sz - 1, 1:sy - 1, 1:sx - 1]
        y0 = 1 + info.location.y * (sy - 2) + 1
        z0 = 1 + info.location.z * (sz - 2) + 1
        zs, ys, xs = min(src.shape[0], Z - z0), min(src.shape[1], Y - y0), min(src.shape[2], X - 2)
        if zs > 0 and ys > 0 and xs > 0:
            full[z0:z0 + zs, y0:y0 + ys, 2:2 + xs] = src[:zs, :ys, :xs]
    return out, (X, Y, Z)


def main(argv=None):
    a = parser().parse_args(argv)
    msg = check_args(a)
    if msg:
        print(msg)
        return 1
    try:
        mesh = load_mesh(a.filename)
    except (OSError, MeshFormatError) as e:
        print(f"{a.filename}: {e}")
        return 1
    node_type = _node_type(a)
    print(f"Starting tests with vox::{_NODE_NAMES[node_type]} @ {api.NODE_BYTES[node_type]} bytes per node.")
    size = a.resolution if a.resolution is not None else float(a.distance)
    vox_res = tuple(a.voxRes) if a.voxRes else api.DEFAULT_VOX
    mat_res = tuple(a.matRes) if a.matRes else api.DEFAULT_MAT
    # The slice tests default both split sizes to (1024, 512) and read the
    # first two values (tests/src/main.cpp:1643-1657, 1824-1837).
    slice_vox = tuple(a.voxRes[:2]) if a.voxRes else (1024, 512)
    slice_mat = tuple(a.matRes[:2]) if a.matRes else (1024, 512)
    try:
        with api.Voxelizer(mesh.vertices, mesh.indices, node_type=node_type, device=a.device) as vz:
            if a.verbose:
                vz.verboseOutput(True)
            if a.materials:
                mats = (1 + np.arange(mesh.n_triangles) % 7).astype(np.uint8)
                vz.setMaterials(mats, 8)
                vz.setMaterialOutput(True)
            t0 = time.perf_counter()
            dims = None
            if a.voxels:
                result, info = vz.voxelizeToRAM(size, vox_res)
            elif a.slice is not None:
                print(f"Slice options: Direction: {a.slice[0]}, slice number: {a.slice[1]}")
                result, info = vz.voxelizeSliceToRAM(size, a.slice[0], a.slice[1], slice_vox, slice_mat)
            elif a.allSlice is not None:
                d = a.allSlice
                dims = vz.getArrayDimensions(size, slice_vox[0], d == 0)
                print(f"Dimensions of big grid: {dims}")
                result = np.zeros(dims[0] * dims[1] * dims[2], dtype=api.NODE_DTYPE[node_type])
                for k in range(dims[d]):
                    sl, _ = vz.voxelizeSliceToRAM(size, d, k, slice_vox, slice_mat)
                    apply_slice(sl, k, result, dims, d)
                info = None
            elif a.multiDevice is not None:
                dy, dz = a.multiDevice
                print(f"DevConf Y: {dy}\nDevConf Z: {dz}")
                result, dims = stitch(vz.voxelizePartsToRAM(True, size, (dy, dz), vox_res, mat_res), dy, dz)
                info = None
            else:
                result, info = vz.voxelizeToNodesToRAM(size, vox_res, mat_res)
            dt = time.perf_counter() - t0
    except api.VxbError as e:
        print(e)
        return 1
    print(f"{mesh.n_vertices} vertices, {mesh.n_triangles} triangles; voxelized in {dt * 1e3:.2f} ms")
    if dims is None:
        dims = info.dims
    for line in summarize(result, dims, not a.voxels, node_type):
        print(line)
    if a.output:
        X, Y, Z = dims
        np.save(a.output, result.reshape(Z, Y, -1) if result.size % (Y * Z) == 0 else result)
        print(f"wrote {a.output}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
