"""Mesh file ingest (the formats the reference's tester reads through VTK,
tests/src/main.cpp:359-417) and the command-line voxelizer.

CPU tests: every writer/reader pair round-trips a closed mesh exactly
(float32 coordinates are written with repr, so ASCII files round-trip
too), polygons are fan-triangulated, and malformed or empty files raise.
The GPU test voxelizes a mesh read from each file format through the
command line and checks the written array against the same mesh
voxelized from memory and against the oracle.
"""

import os
import struct

import numpy as np
import pytest

from voxelizer_b200 import meshio
from voxelizer_b200.scenes import Mesh, icosphere, torus


def _tri_soup(v, f):
    """Triangles as coordinate triples (STL stores no shared vertices)."""
    return np.asarray(v, dtype=np.float32)[np.asarray(f, dtype=np.int64)]


def _write_vtk(path, v, polys):
    with open(path, "w") as fh:
        fh.write("# vtk DataFile Version 3.0\nmesh\nASCII\nDATASET POLYDATA\n")
        fh.write(f"POINTS {len(v)} float\n")
        for x, y, z in np.asarray(v, dtype=np.float64).tolist():
            fh.write(f"{x!r} {y!r} {z!r}\n")
        fh.write(f"POLYGONS {len(polys)} {sum(len(p) + 1 for p in polys)}\n")
        for p in polys:
            fh.write(" ".join(str(x) for x in [len(p), *p]) + "\n")


@pytest.fixture(scope="module")
def sphere():
    return Mesh(*icosphere(2, 0.8, (0.1, -0.2, 0.3)))


@pytest.mark.parametrize("fmt", ["obj", "stl", "ply_bin", "ply_ascii", "vtk"])
def test_round_trip(tmp_path, sphere, fmt):
    v, f = sphere.vertices, sphere.indices
    ext = fmt.split("_")[0]
    path = str(tmp_path / f"m.{ext}")
    if fmt == "obj":
        meshio.save_obj(path, v, f)
    elif fmt == "stl":
        meshio.save_stl(path, v, f)
    elif fmt == "ply_bin":
        meshio.save_ply(path, v, f, binary=True)
    elif fmt == "ply_ascii":
        meshio.save_ply(path, v, f, binary=False)
    else:
        _write_vtk(path, v, f.tolist())
    m = meshio.load_mesh(path)
    assert m.vertices.dtype == np.float32 and m.indices.dtype == np.uint32
    assert m.n_triangles == sphere.n_triangles
    np.testing.assert_array_equal(_tri_soup(m.vertices, m.indices), _tri_soup(v, f))
    if fmt != "stl":
        np.testing.assert_array_equal(m.vertices, v)
        np.testing.assert_array_equal(m.indices, f)


def test_ascii_stl(tmp_path, sphere):
    v, f = sphere.vertices, sphere.indices
    path = str(tmp_path / "a.stl")
    with open(path, "w") as fh:
        fh.write("solid s\n")
        for tri in _tri_soup(v, f).astype(np.float64):
            fh.write("facet normal 0 0 0\n outer loop\n")
            for x, y, z in tri.tolist():
                fh.write(f"  vertex {x!r} {y!r} {z!r}\n")
            fh.write(" endloop\nendfacet\n")
        fh.write("endsolid s\n")
    m = meshio.load_mesh(path)
    np.testing.assert_array_equal(_tri_soup(m.vertices, m.indices), _tri_soup(v, f))


def test_big_endian_ply(tmp_path):
    v = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]], dtype=np.float32)
    path = str(tmp_path / "be.ply")
    with open(path, "wb") as fh:
        fh.write(b"ply\nformat binary_big_endian 1.0\nelement vertex 4\nproperty float x\nproperty float y\n"
                 b"property float z\nelement face 1\nproperty list uchar uint vertex_indices\nend_header\n")
        fh.write(v.astype(">f4").tobytes())
        fh.write(struct.pack(">B4I", 4, 0, 1, 2, 3))
    m = meshio.load_mesh(path)
    np.testing.assert_array_equal(m.vertices, v)
    np.testing.assert_array_equal(m.indices, [[0, 1, 2], [0, 2, 3]])


def test_polygons_fan_triangulated(tmp_path):
    path = str(tmp_path / "quad.obj")
    with open(path, "w") as fh:
        fh.write("# a unit cube as six quads, with texture/normal indices\n")
        for p in [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]:
            fh.write("v %d %d %d\n" % p)
        fh.write("vn 0 0 1\n")
        for q in [(1, 4, 3, 2), (5, 6, 7, 8), (1, 2, 6, 5), (2, 3, 7, 6), (3, 4, 8, 7), (4, 1, 5, 8)]:
            fh.write("f " + " ".join(f"{i}//1" for i in q) + "\n")
    m = meshio.load_mesh(path)
    assert m.n_triangles == 12
    np.testing.assert_array_equal(m.indices[:2], [[0, 3, 2], [0, 2, 1]])
    # negative (relative) OBJ indices name the same vertices
    with open(path, "a") as fh:
        fh.write("f -8 -7 -6\n")
    assert meshio.load_mesh(path).indices[-1].tolist() == [0, 1, 2]


def test_errors(tmp_path):
    bad = str(tmp_path / "m.off")
    open(bad, "w").write("OFF\n")
    with pytest.raises(meshio.MeshFormatError):
        meshio.load_mesh(bad)
    empty = str(tmp_path / "e.obj")
    open(empty, "w").write("v 0 0 0\n")
    with pytest.raises(meshio.MeshFormatError, match="Invalid model data"):
        meshio.load_mesh(empty)
    oob = str(tmp_path / "o.obj")
    open(oob, "w").write("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 9\n")
    with pytest.raises(meshio.MeshFormatError, match="out of range"):
        meshio.load_mesh(oob)
    trunc = str(tmp_path / "t.stl")
    open(trunc, "wb").write(b"\0" * 80 + struct.pack("<I", 5) + b"\0" * 10)
    with pytest.raises(meshio.MeshFormatError):
        meshio.load_mesh(trunc)


def test_cli_argument_errors(tmp_path, capsys, sphere):
    from voxelizer_b200 import cli
    path = str(tmp_path / "s.obj")
    meshio.save_obj(path, sphere.vertices, sphere.indices)
    assert cli.main([path]) == 1
    assert "No resolution or distance" in capsys.readouterr().out
    assert cli.main([str(tmp_path / "missing.obj"), "-r", "32"]) == 1
    a = cli.parser().parse_args([path, "-r", "64", "-L", "-F", "-m", "-V", "64", "32", "32"])
    assert a.resolution == 64 and a.long and a.fcc and a.materials
    assert cli._node_type(a) == cli.api.LONG_FCC and a.voxRes == [64, 32, 32]
    # The tester's checks of the slice and multi-device options.
    for args, msg in ([["-r", "32", "-V", "64", "32"], "--voxRes requires 3 arguments."],
                      [["-r", "32", "-S", "1", "4", "-V", "64", "32", "32"], "--voxRes requires 2 arguments with"],
                      [["-r", "32", "-S", "1", "4", "-M", "64"], "--matRes requires 2 arguments with"],
                      [["-r", "32", "-S", "1"], "--slice requires 2 arguments."],
                      [["-r", "32", "-S", "3", "1"], "The direction of slice is > 2."],
                      [["-r", "32", "-A", "3"], "The direction has to be between 0 and 2."],
                      [["-r", "32", "-D", "2"], "--multiDevice: Device configuration needs two values."]):
        assert cli.main([path, *args]) == 1
        assert msg in capsys.readouterr().out


def test_cli_apply_slice_and_stitch():
    """applySlice and stitchNodeArrays placements (tests/src/main.cpp:1227-1262,
    1396-1434) on labelled arrays."""
    from types import SimpleNamespace as NS
    from voxelizer_b200 import cli
    X, Y, Z = 5, 4, 3
    for d in range(3):
        nodes = np.zeros(X * Y * Z, np.int64)
        n = (X, Y, Z)[d]
        for k in range(n):
            shape = [Z, Y, X]
            shape[2 - d] = 3
            sl = np.full(shape, -1, np.int64)
            idx = [slice(None)] * 3
            idx[2 - d] = 1
            sl[tuple(idx)] = 100 * k + np.arange(sl[tuple(idx)].size).reshape(sl[tuple(idx)].shape)
            cli.apply_slice(sl.reshape(-1), k, nodes, (X, Y, Z), d)
        full = nodes.reshape(Z, Y, X)
        for k in range(n):
            layer = np.take(full, k, axis=2 - d)
            assert np.array_equal(layer.reshape(-1), 100 * k + np.arange(layer.size))
    # Two partitions along y of a 6 x 6 x 4 grid (allocations of 6 x 5 x 4):
    # inner nodes land one step further along every axis.
    parts = []
    for ly in range(2):
        a = np.arange(6 * 5 * 4, dtype=np.int64) + 1000 * ly
        parts.append((a, NS(dims=(6, 5, 4), location=NS(y=ly, z=0))))
    out, dims = cli.stitch(parts, 2, 1)
    assert dims == (6, 8, 4)
    full = out.reshape(4, 8, 6)
    for ly, (a, _) in enumerate(parts):
        src = a.reshape(4, 5, 6)
        for z in range(1, 3):
            for y in range(1, 4):
                for x in range(1, 5):
                    zp, yp, xp = 1 + z, 1 + ly * 3 + y, 1 + x
                    if zp < 4 and yp < 8 and xp < 6:
                        assert full[zp, yp, xp] == src[z, y, x]


# --- GPU: a mesh from a file voxelizes exactly like the same mesh from memory ---

@pytest.mark.gpu
@pytest.mark.parametrize("fmt,flags", [("obj", []), ("stl", ["-L", "-m"]), ("ply", ["-F", "-m", "-d", "0.025"]),
                                       ("vtk", ["-x"]), ("obj", ["-L", "-F", "-d", "0.03"])])
def test_cli_file_matches_memory(tmp_path, fmt, flags):
    import oracle as O
    from voxelizer_b200 import api, cli
    mesh = Mesh(*torus(48, 24, 0.6, 0.25, (0.05, 0.0, -0.1)))
    path = str(tmp_path / f"t.{fmt}")
    {"obj": meshio.save_obj, "stl": meshio.save_stl, "ply": meshio.save_ply}.get(
        fmt, lambda p, v, f: _write_vtk(p, v, f.tolist()))(path, mesh.vertices, mesh.indices)
    out = str(tmp_path / "out.npy")
    args = [path, *flags, "-o", out]
    if "-d" not in flags:   # FCC lattices are sized by cube length only (as in the reference)
        args += ["-r", "96"]
    assert cli.main(args) == 0
    got = np.load(out).reshape(-1)

    a = cli.parser().parse_args(args)
    node_type = cli._node_type(a)
    size = a.resolution if a.resolution is not None else float(a.distance)
    with api.Voxelizer(mesh.vertices, mesh.indices, node_type=node_type) as vz:
        if a.materials:
            vz.setMaterials((1 + np.arange(mesh.n_triangles) % 7).astype(np.uint8), 8)
            vz.setMaterialOutput(True)
        want, info = vz.voxelizeToRAM(size) if a.voxels else vz.voxelizeToNodesToRAM(size)
    np.testing.assert_array_equal(got, want)

    from helpers import masked
    mats = (1 + np.arange(mesh.n_triangles) % 7).astype(np.uint8) if a.materials else None
    om = Mesh(mesh.vertices, mesh.indices, mats, 8 if a.materials else 0)
    ref, _, _ = O.voxelize(om, node_type, int(not a.voxels), int(a.materials), size)
    nodes = not a.voxels
    np.testing.assert_array_equal(masked(node_type, nodes, got), masked(node_type, nodes, ref))


@pytest.mark.gpu
def test_cli_slice_modes(tmp_path):
    """-S, -A and -D give the API's slices and partitions, placed as the
    tester places them."""
    from voxelizer_b200 import api, cli
    mesh = Mesh(*torus(48, 24, 0.6, 0.25, (0.05, 0.0, -0.1)))
    path = str(tmp_path / "t.obj")
    meshio.save_obj(path, mesh.vertices, mesh.indices)
    out = str(tmp_path / "out.npy")
    with api.Voxelizer(mesh.vertices, mesh.indices, node_type=api.LONG) as vz:
        vz.setMaterials((1 + np.arange(mesh.n_triangles) % 7).astype(np.uint8), 8)
        vz.setMaterialOutput(True)
        assert cli.main([path, "-r", "40", "-L", "-m", "-S", "2", "7", "-o", out]) == 0
        want, _ = vz.voxelizeSliceToRAM(40, 2, 7, (1024, 512), (1024, 512))
        np.testing.assert_array_equal(np.load(out).reshape(-1), want)
        for d in range(3):
            assert cli.main([path, "-r", "40", "-L", "-m", "-A", str(d), "-o", out]) == 0
            got = np.load(out).reshape(-1)
            dims = vz.getArrayDimensions(40, 1024, d == 0)
            want = np.zeros(dims[0] * dims[1] * dims[2], np.uint16)
            for k in range(dims[d]):
                cli.apply_slice(vz.voxelizeSliceToRAM(40, d, k, (1024, 512), (1024, 512))[0], k, want, dims, d)
            np.testing.assert_array_equal(got, want)
            assert np.count_nonzero(got)
        assert cli.main([path, "-r", "40", "-L", "-m", "-D", "2", "2", "-o", out]) == 0
        want, _ = cli.stitch(vz.voxelizePartsToRAM(True, 40, (2, 2)), 2, 2)
        np.testing.assert_array_equal(np.load(out).reshape(-1), want)
