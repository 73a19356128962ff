"""Generates the golden fixtures in tests/golden/ from the reference's own CUDA
kernels (hakarlss/Voxelizer src/voxelizer.cu, built unmodified into
oracle/_ref/libvoxref.so by ``make -C oracle ref``) on a B200.

Usage (on a machine with a GPU):

    python tests/golden/make_golden.py --out tests/golden [--only NAME ...]

Every case in cases.py runs twice; ``deterministic`` records whether the two
outputs agree byte for byte (they need not where racing material writes
differ).  Small cases store the whole output array; full-size cases store
SHA-256 digests of the whole output and of the boundary-id field alone, plus
histograms.  Padding bytes inside a node struct (LongFCCNode byte 3,
PartialNode bytes 2-3) are never written deterministically by the reference
and are masked to zero before anything is stored or hashed.
"""

from __future__ import annotations

import argparse
import ctypes
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

import cases as C  # noqa: E402


def load_ref():
    """ref_voxelize_space of oracle/_ref/libvoxref.so: the reference's kernels
    over the whole grid (part NULL) or one device space."""
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libvoxref.so"))
    f = lib.ref_voxelize_space
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint32, ctypes.c_double,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p,
                  ctypes.c_uint32, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_int,
                  ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_void_p]
    lib.ref_last_error.restype = ctypes.c_char_p
    f.last_error = lambda: lib.ref_last_error().decode()
    return f


def padding_mask(c):
    """Mask of meaningful bits for one element of the output dtype."""
    if not c["nodes"]:
        return None
    t = c["node_type"]
    if t == C.LONG_FCC:
        return np.uint32(0x00FFFFFF)
    if t == C.PARTIAL:
        return np.uint64(0xFFFFFFFF0000FFFF)
    return None


def bid_of(c, a):
    t = c["node_type"]
    if t == C.SHORT:
        return a & 31
    if t == C.LONG:
        return a & 0xFF
    if t == C.PARTIAL:
        return a & 0xFF
    if t == C.SHORT_FCC:
        return a & 4095
    if t == C.LONG_FCC:
        return a & 0xFFFF
    raise ValueError(t)


def mat_of(c, a):
    t = c["node_type"]
    if t == C.SHORT:
        return a >> 5
    if t == C.LONG:
        return a >> 8
    if t == C.PARTIAL:
        return (a >> 8) & 0xFF
    if t == C.SHORT_FCC:
        return a >> 12
    if t == C.LONG_FCC:
        return (a >> 16) & 0xFF
    raise ValueError(t)


def run_case(f, c):
    m = C.mesh(c["mesh"])
    dims = (ctypes.c_uint32 * 3)()
    vs = (ctypes.c_uint32 * 3)(*c["vox"])
    ms = (ctypes.c_uint32 * 3)(*c["mat"])
    elapsed = ctypes.c_double(0.0)
    md = 0 if c["by_cube"] else int(c["size"])
    cl = float(c["size"]) if c["by_cube"] else 0.0
    mats = m.materials if m.materials is not None else np.zeros(m.n_triangles, np.uint8)
    args = [c["node_type"], c["nodes"], c["materials"], int(c["by_cube"]), md, cl, vs, ms,
            m.vertices.ctypes.data, m.n_vertices, m.indices.ctypes.data, m.n_triangles,
            mats.ctypes.data, m.n_materials]
    rot = int(C.turned(c))
    rc = f(*args, None, rot, None, 0, dims, None)
    if rc != 0:
        raise RuntimeError(f"{c['name']}: plan failed rc={rc}")
    part, oob = None, False
    if c.get("space"):
        fcc = c["nodes"] and c["node_type"] in (C.SHORT_FCC, C.LONG_FCC)   # FCC arrays double z
        res_y, res_z = int(dims[1]) - 2, (int(dims[2]) // 2 if fcc else int(dims[2])) - 2
        part = (ctypes.c_uint32 * 4)(*C.partition(c, res_y, res_z))
        oob = C.slice_oob(c, res_y, res_z)
        rc = f(*args, part, rot, None, 0, dims, None)
        if rc != 0:
            raise RuntimeError(f"{c['name']}: plan failed rc={rc}")
    args += [part, rot]
    dt = C.out_dtype(c)
    n = int(dims[0]) * int(dims[1]) * int(dims[2])
    count = n // 32 if not c["nodes"] else n
    outs, times = [], []
    for _ in range(2):
        out = np.empty(count, dtype=dt)
        rc = f(*args, out.ctypes.data, out.nbytes, dims, ctypes.byref(elapsed))
        if rc != 0:
            raise RuntimeError(f"reference failed rc={rc}: {f.last_error()}")
        pm = padding_mask(c)
        if pm is not None:
            out &= pm
        if oob:   # sliceOOB: the reference zeroes the slice array (src/host_side.cpp:1225-1236)
            out[:] = 0
        outs.append(out)
        times.append(elapsed.value)
    return m, (int(dims[0]), int(dims[1]), int(dims[2])), outs, times


def summarize(c, out):
    info = {"sha256": hashlib.sha256(out.tobytes()).hexdigest(), "count": int(out.size)}
    if c["nodes"]:
        bid = bid_of(c, out)
        mat = mat_of(c, out)
        info["bid_sha256"] = hashlib.sha256(bid.astype(np.uint32).tobytes()).hexdigest()
        info["n_solid"] = int(np.count_nonzero(bid))
        if c["node_type"] in (C.SHORT_FCC, C.LONG_FCC):
            info["bid_hist"] = np.bincount(np.bitwise_count(bid.astype(np.uint16)), minlength=13).tolist()
        else:
            info["bid_hist"] = np.bincount(bid.astype(np.int64), minlength=28).tolist()
        info["mat_hist"] = np.bincount(mat.astype(np.int64), minlength=2).tolist()
    else:
        info["n_set_bits"] = int(np.bitwise_count(out).sum())
    return info


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--only", nargs="*")
    args = ap.parse_args()
    f = load_ref()
    os.makedirs(args.out, exist_ok=True)
    index_path = os.path.join(args.out, "index.json")
    index = json.load(open(index_path)) if os.path.exists(index_path) else {}
    for c in C.CASES:
        if args.only and c["name"] not in args.only:
            continue
        t0 = time.time()
        try:
            m, dims, outs, times = run_case(f, c)
        except RuntimeError as e:
            # Recorded, not fatal: e.g. a reference kernel that cannot launch.
            index[c["name"]] = {"ref_error": str(e), "case": {k: (list(v) if isinstance(v, tuple) else v)
                                                              for k, v in c.items()}}
            print(f"{c['name']}: {e}", flush=True)
            json.dump(index, open(index_path, "w"), indent=1, sort_keys=True)
            continue
        det = bool(np.array_equal(outs[0], outs[1]))
        entry = {"dims": dims, "mesh_sha256": C.mesh_digest(m), "deterministic": det,
                 "ref_ms": times, "n_triangles": m.n_triangles, "n_vertices": m.n_vertices,
                 "case": {k: (list(v) if isinstance(v, tuple) else v) for k, v in c.items()}}
        entry.update(summarize(c, outs[0]))
        if not det and c["nodes"]:
            entry["bid_deterministic"] = bool(np.array_equal(bid_of(c, outs[0]), bid_of(c, outs[1])))
            entry["n_diff"] = int(np.count_nonzero(outs[0] != outs[1]))
        if c["store"] == "full":
            extra = {} if det else {"out2": outs[1]}
            np.savez_compressed(os.path.join(args.out, c["name"] + ".npz"), out=outs[0], **extra)
        index[c["name"]] = entry
        print(f"{c['name']}: dims={dims} det={det} ref_ms={[round(t, 2) for t in times]} "
              f"({time.time() - t0:.1f}s)", flush=True)
        json.dump(index, open(index_path, "w"), indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
