"""Triangle-mesh file readers: OBJ, STL (binary and ASCII), PLY (ASCII and
binary), legacy VTK polydata (ASCII).

These are the formats the reference's tester loads through VTK
(tests/src/main.cpp:359-417, loadModel 911-955): vertices become float32
xyz triples, faces vertex-index triples.  Polygons with more than three
vertices are split into a fan of triangles (the tester's loadModel expects
triangles only).  Vertex sharing does not change a voxelization: the
bounding box and every triangle's coordinates are the same whether
duplicate vertices are merged or not, so STL facets keep their own three
vertices each.
"""

from __future__ import annotations

import os
import struct

import numpy as np

from .scenes import Mesh


class MeshFormatError(ValueError):
    pass


def _fan(polys):
    """(vertex index lists) -> uint32 triangles (fan from the first vertex)."""
    tris = []
    for p in polys:
        if len(p) < 3:
            raise MeshFormatError(f"face with {len(p)} vertices")
        for k in range(1, len(p) - 1):
            tris.append((p[0], p[k], p[k + 1]))
    return np.asarray(tris, dtype=np.uint32).reshape(-1, 3)


def load_obj(path):
    verts, polys = [], []
    with open(path, "r", errors="replace") as fh:
        for line in fh:
            parts = line.split()
            if not parts:
                continue
            if parts[0] == "v" and len(parts) >= 4:
                verts.append((float(parts[1]), float(parts[2]), float(parts[3])))
            elif parts[0] == "f":
                face = []
                for tok in parts[1:]:
                    i = int(tok.split("/")[0])
                    face.append(i - 1 if i > 0 else len(verts) + i)   # negative: relative to the end
                polys.append(face)
    return np.asarray(verts, dtype=np.float32).reshape(-1, 3), _fan(polys)


def load_stl(path):
    with open(path, "rb") as fh:
        data = fh.read()
    if len(data) >= 84:
        n = struct.unpack_from("<I", data, 80)[0]
        if 84 + 50 * n == len(data):
            rec = np.frombuffer(data, dtype=np.dtype([("n", "<f4", 3), ("v", "<f4", (3, 3)), ("a", "<u2")]),
                                count=n, offset=84)
            v = np.ascontiguousarray(rec["v"].reshape(-1, 3), dtype=np.float32)
            return v, np.arange(3 * n, dtype=np.uint32).reshape(-1, 3)
    text = data.decode("ascii", errors="replace")
    if not text.lstrip().startswith("solid"):
        raise MeshFormatError("neither binary nor ASCII STL")
    verts = [tuple(float(x) for x in line.split()[1:4]) for line in text.splitlines()
             if line.strip().startswith("vertex")]
    if len(verts) % 3:
        raise MeshFormatError("ASCII STL facets must have three vertices")
    v = np.asarray(verts, dtype=np.float32).reshape(-1, 3)
    return v, np.arange(v.shape[0], dtype=np.uint32).reshape(-1, 3)


_PLY_TYPES = {"char": "i1", "int8": "i1", "uchar": "u1", "uint8": "u1", "short": "i2", "int16": "i2",
              "ushort": "u2", "uint16": "u2", "int": "i4", "int32": "i4", "uint": "u4", "uint32": "u4",
              "float": "f4", "float32": "f4", "double": "f8", "float64": "f8"}


def load_ply(path):
    with open(path, "rb") as fh:
        if fh.readline().strip() != b"ply":
            raise MeshFormatError("not a PLY file")
        fmt = None
        elements = []   # [name, count, [(prop, type) or (prop, ("list", count_t, item_t))]]
        while True:
            line = fh.readline()
            if not line:
                raise MeshFormatError("PLY header without end_header")
            parts = line.decode("ascii", errors="replace").split()
            if not parts:
                continue
            if parts[0] == "format":
                fmt = parts[1]
            elif parts[0] == "element":
                elements.append([parts[1], int(parts[2]), []])
            elif parts[0] == "property":
                if parts[1] == "list":
                    elements[-1][2].append((parts[4], ("list", _PLY_TYPES[parts[2]], _PLY_TYPES[parts[3]])))
                else:
                    elements[-1][2].append((parts[2], _PLY_TYPES[parts[1]]))
            elif parts[0] == "end_header":
                break
        body = fh.read()
    if fmt not in ("ascii", "binary_little_endian", "binary_big_endian"):
        raise MeshFormatError(f"unsupported PLY format {fmt}")
    verts, polys = None, []
    if fmt == "ascii":
        tokens = body.split()
        pos = 0
        for name, count, props in elements:
            rows = []
            for _ in range(count):
                row = {}
                for pname, ptype in props:
                    if isinstance(ptype, tuple):
                        k = int(tokens[pos])
                        row[pname] = [int(t) for t in tokens[pos + 1:pos + 1 + k]]
                        pos += 1 + k
                    else:
                        row[pname] = float(tokens[pos])
                        pos += 1
                rows.append(row)
            if name == "vertex":
                verts = np.asarray([(r["x"], r["y"], r["z"]) for r in rows], dtype=np.float32)
            elif name == "face":
                key = "vertex_indices" if rows and "vertex_indices" in rows[0] else "vertex_index"
                polys = [r[key] for r in rows]
    else:
        end = "<" if fmt == "binary_little_endian" else ">"
        off = 0
        for name, count, props in elements:
            if all(not isinstance(t, tuple) for _, t in props):
                dt = np.dtype([(p, end + t) for p, t in props])
                arr = np.frombuffer(body, dtype=dt, count=count, offset=off)
                off += dt.itemsize * count
                if name == "vertex":
                    verts = np.stack([arr["x"], arr["y"], arr["z"]], axis=1).astype(np.float32)
                continue
            # Elements with list properties: walk record by record.
            rows = []
            for _ in range(count):
                row = {}
                for pname, ptype in props:
                    if isinstance(ptype, tuple):
                        ct = np.dtype(end + ptype[1])
                        k = int(np.frombuffer(body, dtype=ct, count=1, offset=off)[0])
                        off += ct.itemsize
                        it = np.dtype(end + ptype[2])
                        row[pname] = np.frombuffer(body, dtype=it, count=k, offset=off).astype(np.int64).tolist()
                        off += it.itemsize * k
                    else:
                        t = np.dtype(end + ptype)
                        row[pname] = np.frombuffer(body, dtype=t, count=1, offset=off)[0]
                        off += t.itemsize
                rows.append(row)
            if name == "face":
                key = "vertex_indices" if rows and "vertex_indices" in rows[0] else "vertex_index"
                polys = [r[key] for r in rows]
    if verts is None:
        raise MeshFormatError("PLY file without vertices")
    return verts.reshape(-1, 3), _fan(polys)


def load_vtk(path):
    """Legacy VTK ASCII POLYDATA with POINTS and POLYGONS."""
    with open(path, "r", errors="replace") as fh:
        tokens = fh.read().split()
    if "POLYDATA" not in tokens:
        raise MeshFormatError("only legacy ASCII POLYDATA files are read")
    i = tokens.index("POINTS")
    n = int(tokens[i + 1])
    verts = np.asarray(tokens[i + 3:i + 3 + 3 * n], dtype=np.float64).astype(np.float32).reshape(-1, 3)
    polys = []
    if "POLYGONS" in tokens:
        j = tokens.index("POLYGONS")
        count = int(tokens[j + 1])
        pos = j + 3
        for _ in range(count):
            k = int(tokens[pos])
            polys.append([int(t) for t in tokens[pos + 1:pos + 1 + k]])
            pos += 1 + k
    return verts, _fan(polys)


_LOADERS = {".obj": load_obj, ".stl": load_stl, ".ply": load_ply, ".vtk": load_vtk}


def load_mesh(path) -> Mesh:
    """Reads a triangle mesh by file extension (.obj, .stl, .ply, .vtk)."""
    ext = os.path.splitext(str(path))[1].lower()
    if ext not in _LOADERS:
        raise MeshFormatError(f"unsupported mesh file type {ext!r}")
    v, f = _LOADERS[ext](path)
    if f.shape[0] == 0:
        raise MeshFormatError("Invalid model data given")   # the tester's message for an empty model
    if f.size and int(f.max()) >= v.shape[0]:
        raise MeshFormatError("face index out of range")
    return Mesh(v, f, None, 0, os.path.basename(str(path)))


def save_obj(path, vertices, indices):
    """Writes an OBJ file (for tests and examples)."""
    with open(path, "w") as fh:
        for x, y, z in np.asarray(vertices, dtype=np.float64).reshape(-1, 3).tolist():
            fh.write(f"v {x!r} {y!r} {z!r}\n")
        for a, b, c in (np.asarray(indices, dtype=np.int64).reshape(-1, 3) + 1).tolist():
            fh.write(f"f {a} {b} {c}\n")


def save_stl(path, vertices, indices):
    """Writes a binary STL file."""
    v = np.asarray(vertices, dtype=np.float32).reshape(-1, 3)
    f = np.asarray(indices).reshape(-1, 3)
    rec = np.zeros(f.shape[0], dtype=np.dtype([("n", "<f4", 3), ("v", "<f4", (3, 3)), ("a", "<u2")]))
    rec["v"] = v[f]
    with open(path, "wb") as fh:
        fh.write(b"\0" * 80)
        fh.write(struct.pack("<I", f.shape[0]))
        fh.write(rec.tobytes())


def save_ply(path, vertices, indices, binary=True):
    """Writes a PLY file (binary little endian or ASCII)."""
    v = np.asarray(vertices, dtype=np.float32).reshape(-1, 3)
    f = np.asarray(indices, dtype=np.int32).reshape(-1, 3)
    head = ("ply\nformat " + ("binary_little_endian" if binary else "ascii") + " 1.0\n"
            f"element vertex {v.shape[0]}\nproperty float x\nproperty float y\nproperty float z\n"
            f"element face {f.shape[0]}\nproperty list uchar int vertex_indices\nend_header\n")
    with open(path, "wb") as fh:
        fh.write(head.encode("ascii"))
        if binary:
            fh.write(v.astype("<f4").tobytes())
            rec = np.zeros(f.shape[0], dtype=np.dtype([("k", "u1"), ("i", "<i4", 3)]))
            rec["k"] = 3
            rec["i"] = f
            fh.write(rec.tobytes())
        else:
            for x, y, z in v.astype(np.float64).tolist():
                fh.write(f"{x!r} {y!r} {z!r}\n".encode())
            for a, b, c in f.tolist():
                fh.write(f"3 {a} {b} {c}\n".encode())
