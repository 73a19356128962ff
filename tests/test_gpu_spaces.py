"""Device spaces: slices (voxelizeSlice, src/host_side.cpp:1927-2262) and
devConfig partitions (voxelizeEntry / voxelizeWorker, 782-1236).

The golden cases in test_gpu_parity pin single slices and partitions
against the reference's kernels; here the CUDA path is swept over many
slices and partition layouts against the oracle (bit-exact), and argument
errors are checked (CPU).
"""

import numpy as np
import pytest

import cases as C
import oracle as O
from helpers import masked
from voxelizer_b200._lib import VxbError
from voxelizer_b200.api import LONG, LONG_FCC, SHORT, SHORT_FCC, Voxelizer


def _oracle_space(m, node_type, nodes, size, vox, mat, part, oob=False, rotate_x=False):
    out, info, _ = O.voxelize(m, node_type, nodes, int(nodes and m.materials is not None), size, vox, mat,
                              part=part, rotate_x=rotate_x)
    if oob:
        out[:] = 0
    return masked(node_type, nodes, out), info


def test_slice_argument_errors():
    m = C.mesh("torus")
    with Voxelizer(m.vertices, m.indices, node_type=LONG) as v:
        info = v.planSlice(120, 0, 5)   # x: the turned grid sliced along its y, turned back
        assert info.dims[0] == 3 and tuple(info.partition)[:2] == (4, 5)
        turned = v.getArrayDimensions(120, 1024, True)
        assert (info.dims[1], info.dims[2]) == (turned[1], turned[2])
        with pytest.raises(VxbError, match="EINVAL"):
            v.planSlice(120, 3, 5)
        info = v.planSlice(120, 1, 7)
        assert info.dims[1] == 3 and tuple(info.partition)[:2] == (6, 7)
        info = v.planSlice(120, 2, 7)
        assert info.dims[2] == 3 and tuple(info.partition)[2:] == (6, 7)
        with pytest.raises(VxbError, match="EINVAL"):
            v.planParts(1, 120, (0, 2))
        with pytest.raises(VxbError, match="EINVAL"):
            v.planParts(1, 120, (200, 1))   # more partitions than rows
        infos = v.planParts(1, 120, (3, 2))
        assert [(i.location.y, i.location.z) for i in infos] == [(0, 0), (1, 0), (2, 0), (0, 1), (1, 1), (2, 1)]
        parts = [tuple(i.partition) for i in infos]
        full = v.plan(1, 120)
        assert parts[0][0] == 0 and parts[2][1] == full.resolution.y and parts[5][3] == full.resolution.z
    with Voxelizer(m.vertices, m.indices, node_type=SHORT_FCC) as v:
        full = v.plan(1, 1.0 / 64.0)
        info = v.planSlice(1.0 / 64.0, 0, 5)   # FCC along x: the turned lattice turned back
        turned = v.getArrayDimensions(1.0 / 64.0, 1024, True)
        assert info.dims == (6, turned[1], turned[2])
        info = v.planSlice(1.0 / 64.0, 1, 5)   # FCC: x and z doubled, three voxel rows along y
        assert info.dims == (full.dims[0], 3, full.dims[2])
        info = v.planSlice(1.0 / 64.0, 2, 5)
        assert info.dims == (full.dims[0], full.dims[1], 6)
        infos = v.planParts(1, 1.0 / 64.0, (2, 1))
        assert sum(i.dims[1] - 2 for i in infos) == full.dims[1] - 2


@pytest.mark.gpu
@pytest.mark.parametrize("direction", [0, 1, 2])
def test_slice_sweep_matches_oracle(direction):
    m = C.mesh("torus")
    size, vox, mat = 64, (1024, 512, 512), (512, 512, 512)
    rot = direction == 0   # slices along x cut the turned grid along its y
    res = O.plan(m, LONG, 1, size, vox, rotate_x=rot).resolution
    ry, rz = int(res[1]), int(res[2])
    n = rz if direction == 2 else ry
    with Voxelizer(m.vertices, m.indices, node_type=LONG) as v:
        v.setMaterials(m.materials, m.n_materials)
        for s in [0, 1, 2, n // 3, n // 2, n - 1, n, n + 1]:
            got, info = v.voxelizeSliceToRAM(size, direction, s, vox, mat)
            s0 = 0 if (s == 0 or s > n) else s - 1
            part = (0, ry, s0, s0 + 1) if direction == 2 else (s0, s0 + 1, 0, rz)
            want, _ = _oracle_space(m, LONG, 1, size, vox, mat, part, oob=(s == 0 or s > n), rotate_x=rot)
            assert np.array_equal(got, want), f"slice {s} along {direction}"
            X, Y, Z = info.dims
            g = got.reshape(Z, Y, X)
            outer = g[:, :, [0, 2]] if direction == 0 else g[:, [0, 2], :] if direction == 1 else g[[0, 2], :, :]
            assert not outer.any(), "outer layers of a slice are zero"


@pytest.mark.gpu
@pytest.mark.parametrize("dev", [(2, 1), (1, 2), (3, 2), (4, 3)])
@pytest.mark.parametrize("nodes", [1, 0])
def test_partitions_match_oracle(dev, nodes):
    m = C.mesh("room_lite")
    size, vox, mat = 120, (1024, 24, 20), (512, 512, 512)
    with Voxelizer(m.vertices, m.indices, node_type=SHORT) as v:
        v.setMaterials(np.minimum(m.materials, 7), 8)
        res = v.voxelizePartsToRAM(nodes, size, dev, vox, mat)
        full = v.plan(nodes, size, vox, mat)
    assert len(res) == dev[0] * dev[1]
    ys = C.split_parts(full.resolution.y, dev[0])
    zs = C.split_parts(full.resolution.z, dev[1])
    mm = m.__class__(m.vertices, m.indices, np.minimum(m.materials, 7), 8)
    for k, (got, info) in enumerate(res):
        y, z = k % dev[0], k // dev[0]
        part = (ys[y][0], ys[y][1], zs[z][0], zs[z][1])
        assert tuple(info.partition) == part and (info.location.y, info.location.z) == (y, z)
        want, oi = _oracle_space(mm, SHORT, nodes, size, vox, mat, part)
        assert info.dims == tuple(oi.dims)
        assert np.array_equal(got, want), f"partition {k} of {dev}"


@pytest.mark.gpu
@pytest.mark.parametrize("node_type", [SHORT_FCC, LONG_FCC])
def test_fcc_spaces_match_oracle(node_type):
    """FCC lattices in device spaces: each sub-lattice voxelized over the
    extended partition from its shifted corner, the faces of an allocation
    with neighbours zeroed two node layers deep along x and z."""
    m = C.mesh("ico4")
    mats = (1 + np.arange(m.n_triangles) % 9).astype(np.uint8)
    mm = m.__class__(m.vertices, m.indices, mats, 10)
    size, vox, mat = C.FCC_A, (1024, 512, 512), (512, 512, 512)
    res = O.plan(mm, node_type, 1, size, vox).resolution
    ry, rz = int(res[1]), int(res[2])
    tres = O.plan(mm, node_type, 1, size, vox, rotate_x=True).resolution   # slices along x cut the turned grid
    with Voxelizer(mm.vertices, mm.indices, node_type=node_type) as v:
        v.setMaterials(mats, 10)
        for direction, n in ((1, ry), (2, rz), (0, int(tres[1]))):
            rot = direction == 0
            sy, sz = (int(tres[1]), int(tres[2])) if rot else (ry, rz)
            for s in [0, 1, n // 2, n, n + 1]:
                got, info = v.voxelizeSliceToRAM(size, direction, s, vox, mat)
                s0 = 0 if (s == 0 or s > n) else s - 1
                part = (0, sy, s0, s0 + 1) if direction == 2 else (s0, s0 + 1, 0, sz)
                want, oi = _oracle_space(mm, node_type, 1, size, vox, mat, part, oob=(s == 0 or s > n),
                                         rotate_x=rot)
                assert info.dims == tuple(oi.dims)
                assert np.array_equal(masked(node_type, 1, got), want), f"slice {s} along {direction}"
        for dev in [(2, 2), (3, 1)]:
            ys, zs = C.split_parts(ry, dev[0]), C.split_parts(rz, dev[1])
            for k, (got, info) in enumerate(v.voxelizePartsToRAM(1, size, dev, vox, mat)):
                y, z = k % dev[0], k // dev[0]
                part = (ys[y][0], ys[y][1], zs[z][0], zs[z][1])
                want, oi = _oracle_space(mm, node_type, 1, size, vox, mat, part)
                assert info.dims == tuple(oi.dims)
                assert np.array_equal(masked(node_type, 1, got), want), f"partition {k} of {dev}"
