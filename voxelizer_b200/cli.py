"""Command-line voxelizer mirroring the reference's tester
(tests/src/main.cpp:197-450, initTests 1520-1580).

    python -m voxelizer_b200.cli MODEL.(obj|stl|ply|vtk) -r 256 [-x] [-m] [-L|-P|-F] \
        [-V X Y Z] [-M X Y Z] [-v] [-o OUT.npy]

Options keep the tester's letters and meaning: ``-r`` voxels along the
longest side, ``-d`` distance between voxel centres, ``-x`` plain voxel
output instead of nodes, ``-m`` materials with the tester's mapping
(triangle i gets material 1 + i % 7, eight unique materials, material
output on), ``-L`` / ``-P`` / ``-F`` the node type (``-L -F`` is the long FCC
node), ``-V`` / ``-M`` the internal voxel / material split resolutions,
``-v`` verbose.  The tester renders the result with VTK; here the result is
written as a numpy array (``-o``) and summarised on stdout.  The tester's
slice (``-S``, ``-A``) and simulated multi-device (``-D``) modes are not
provided by this command.
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
    p.add_argument("-V", "--voxRes", type=int, nargs=3, metavar=("X", "Y", "Z"),
                   help="Internal voxelization dimensions.")
    p.add_argument("-M", "--matRes", type=int, nargs=3, metavar=("X", "Y", "Z"),
                   help="Internal material voxelization dimensions.")
    p.add_argument("-v", "--verbose", action="store_true", help="Prints detailed information about the voxelization.")
    p.add_argument("-o", "--output", help="Write the result array to this .npy file.")
    p.add_argument("--device", type=int, default=0, help="CUDA device.")
    return p


_BID = {api.SHORT: (0x1F, 5, 0x7), api.LONG: (0xFF, 8, 0xFF), api.PARTIAL: (0xFF, 8, 0xFF),
        api.SHORT_FCC: (0xFFF, 12, 0xF), api.LONG_FCC: (0xFFFF, 16, 0xFF)}


def summarize(result, info, nodes, node_type):
    """Text lines: grid size, solid count, boundary-id and material histograms."""
    X, Y, Z = info.dims
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


def main(argv=None):
    a = parser().parse_args(argv)
    if a.resolution is None and a.distance is None:
        print("No resolution or distance was given.")
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
    try:
        with api.Voxelizer(mesh.vertices, mesh.indices, node_type=node_type, device=a.device) as vz:
            if a.verbose:
                vz.verboseOutput(True)
            if a.materials:
                mats = (1 + np.arange(mesh.n_triangles) % 7).astype(np.uint8)
                vz.setMaterials(mats, 8)
                vz.setMaterialOutput(True)
            t0 = time.perf_counter()
            if a.voxels:
                result, info = vz.voxelizeToRAM(size, vox_res)
            else:
                result, info = vz.voxelizeToNodesToRAM(size, vox_res, mat_res)
            dt = time.perf_counter() - t0
    except api.VxbError as e:
        print(e)
        return 1
    print(f"{mesh.n_vertices} vertices, {mesh.n_triangles} triangles; voxelized in {dt * 1e3:.2f} ms")
    for line in summarize(result, info, not a.voxels, node_type):
        print(line)
    if a.output:
        X, Y, Z = info.dims
        np.save(a.output, result.reshape(Z, Y, -1) if result.size % (Y * Z) == 0 else result)
        print(f"wrote {a.output}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
