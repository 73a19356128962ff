"""The C++ drop-in front end (include/vox/voxelizer.h) compiled into a
program the way a user of the reference would write it, run on the GPU, and
compared with the C ABI results."""

import os
import subprocess

import numpy as np
import pytest

from voxelizer_b200 import scenes
from voxelizer_b200.api import LONG, SHORT, Voxelizer

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_cpp_front_end(tmp_path):
    exe = tmp_path / "api_drop_in"
    lib = os.path.join(ROOT, "voxelizer_b200")
    subprocess.run(["nvcc", "-std=c++17", "-O2", "-Wno-deprecated-gpu-targets", "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "api_drop_in.cpp"), "-L" + lib, "-lvxb",
                    "-Xlinker", "-rpath=" + lib, "-o", str(exe)], check=True)
    v, f = scenes.icosphere(3, 0.4, (0.5, 0.5, 0.5))
    mats = (1 + np.arange(f.shape[0]) % 7).astype(np.uint8)
    mesh = tmp_path / "mesh.bin"
    with open(mesh, "wb") as fh:
        fh.write(np.array([v.shape[0], f.shape[0]], np.uint32).tobytes())
        fh.write(v.tobytes())
        fh.write(f.astype(np.uint32).tobytes())
        fh.write(mats.tobytes())
    out = subprocess.run([str(exe), str(mesh), str(tmp_path / "r")], capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    raw = open(tmp_path / "r_nodes.bin", "rb").read()
    dims = tuple(np.frombuffer(raw[:12], np.uint32))
    nodes = np.frombuffer(raw[12:], np.uint16)
    with Voxelizer(v, f, mats, 8, node_type=LONG) as vx:
        want, info = vx.voxelizeToNodesToRAM(80)
    assert dims == info.dims
    assert np.array_equal(nodes, want)
    assert np.array_equal(np.fromfile(tmp_path / "r_nodes_dev.bin", np.uint16), want)
    with Voxelizer(v, f, mats, 8, node_type=LONG) as vx:
        wslice, sinfo = vx.voxelizeSliceToRAM(80, 1, 20)
        wparts = vx.voxelizePartsToRAM(1, 80, (2, 2))
        wsim = vx.voxelizePartsToRAM(1, 80, (2, 1))
    raw = open(tmp_path / "r_slice.bin", "rb").read()
    assert tuple(np.frombuffer(raw[:12], np.uint32)) == sinfo.dims
    assert np.array_equal(np.frombuffer(raw[12:], np.uint16), wslice)
    for fname, want_parts in (("r_parts.bin", wparts), ("r_sim.bin", wsim)):
        raw = open(tmp_path / fname, "rb").read()
        pos = 0
        for want_arr, want_info in want_parts:
            dims = tuple(np.frombuffer(raw[pos:pos + 12], np.uint32))
            loc = tuple(np.frombuffer(raw[pos + 12:pos + 24], np.uint32))
            pos += 24
            assert dims == want_info.dims
            assert loc == (want_info.location.x, want_info.location.y, want_info.location.z)
            n = dims[0] * dims[1] * dims[2]
            assert np.array_equal(np.frombuffer(raw[pos:pos + 2 * n], np.uint16), want_arr)
            pos += 2 * n
        assert pos == len(raw)
    raw = open(tmp_path / "r_bits.bin", "rb").read()
    with Voxelizer(v, f, node_type=SHORT) as vx:
        wbits, binfo = vx.voxelizeToRAM(80)
    assert tuple(np.frombuffer(raw[:12], np.uint32)) == binfo.dims
    assert np.array_equal(np.frombuffer(raw[12:], np.uint32), wbits)
