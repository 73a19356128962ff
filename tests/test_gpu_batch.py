"""Batches (vxb_batch_*): every mesh of a batch must come out exactly as its
single-mesh call, for each node family, with and without CUDA graph replay,
and on repeated runs."""

import numpy as np
import pytest

import cases as C
from voxelizer_b200 import scenes
from voxelizer_b200.api import LONG, LONG_FCC, PARTIAL, SHORT, SHORT_FCC, Voxelizer, VoxelizerBatch

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _meshes():
    """A mix of sizes and shapes: small spheres, a torus, the stress scene
    with slivers and snapped vertices, a small room."""
    out = []
    for lvl, r, c in ((2, 0.3, (0.5, 0.4, 0.5)), (4, 0.45, (0.1, 0.2, 0.3)), (3, 0.2, (0.0, 0.0, 0.0))):
        v, f = scenes.icosphere(lvl, r, c)
        m = (1 + np.arange(f.shape[0]) % 5).astype(np.uint8)
        out.append(scenes.Mesh(v, f, m, 6, f"ico{lvl}"))
    out.append(C.mesh("torus"))
    out.append(C.mesh("stress"))
    out.append(C.mesh("room_lite"))
    return out


MAX_MATERIAL = {SHORT: 7, LONG: 255, PARTIAL: 255, SHORT_FCC: 15, LONG_FCC: 255}


def _single(mesh, node_type, nodes, size, vox, mat, materials=True):
    v = Voxelizer(mesh.vertices, mesh.indices, node_type=node_type)
    if materials and nodes:
        mats = (mesh.materials.astype(np.int64) % (MAX_MATERIAL[node_type] + 1)).astype(np.uint8)
        v.setMaterials(mats, int(mats.max()) + 1)
    info = v.plan(nodes, size, vox, mat)
    out = torch.zeros(int(info.bytes), dtype=torch.uint8, device="cuda")
    v.voxelize_device(nodes, size, out, vox, mat)
    torch.cuda.synchronize()
    return v, info, out


def _check_batch(node_type, nodes, sizes, vox=(1024, 512, 512), mat=(512, 512, 512), graph=False, materials=True):
    meshes = _meshes()
    singles = [_single(m, node_type, nodes, s, vox, mat, materials) for m, s in zip(meshes, sizes)]
    with VoxelizerBatch() as b:
        outs = []
        for (v, info, ref), s in zip(singles, sizes):
            out = torch.full((int(info.bytes),), 0xA5, dtype=torch.uint8, device="cuda")
            got = b.add(v, nodes, s, out, vox, mat)
            assert got.dims == info.dims and got.bytes == info.bytes
            outs.append(out)
        for rep in range(2):
            b.run(graph=graph)
            torch.cuda.synchronize()
            for (v, info, ref), out, m in zip(singles, outs, meshes):
                assert torch.equal(out, ref), f"{m.name}: batch result differs (run {rep}, graph={graph})"
            assert b.last_launch_count() > 0
            for out in outs:
                out.fill_(0x5A)
    for v, _, _ in singles:
        v.close()


@pytest.mark.parametrize("graph", [False, True])
def test_batch_long_nodes(graph):
    _check_batch(LONG, 1, [40, 96, 1.0 / 64.0, 80, 1.0 / 128.0, 120], graph=graph)


def test_batch_long_nodes_small_splits():
    # Several pruning subspaces and material slices per mesh.
    _check_batch(LONG, 1, [40, 96, 1.0 / 64.0, 80, 1.0 / 128.0, 120], vox=(64, 32, 48), mat=(40, 24, 32))


def test_batch_short_nodes_no_materials():
    _check_batch(SHORT, 1, [33, 70, 1.0 / 50.0, 64, 1.0 / 100.0, 90], materials=False)


def test_batch_partial_nodes():
    _check_batch(PARTIAL, 1, [32, 48, 1.0 / 40.0, 40, 1.0 / 64.0, 64])


@pytest.mark.parametrize("node_type", [SHORT_FCC, LONG_FCC])
def test_batch_fcc(node_type):
    a = 4.0 ** (1.0 / 3.0)
    _check_batch(node_type, 1, [a / 40, a / 64, a / 50, a / 48, a / 100, a / 3.0], graph=True)


def test_batch_plain_bits():
    _check_batch(LONG, 0, [40, 96, 1.0 / 64.0, 80, 1.0 / 128.0, 120], graph=True)


def test_batch_rejects_mixed_node_types():
    m = _meshes()[0]
    with Voxelizer(m.vertices, m.indices, node_type=LONG) as a, Voxelizer(m.vertices, m.indices,
                                                                          node_type=SHORT) as c:
        ia = a.plan(1, 32)
        ic = c.plan(1, 32)
        oa = torch.empty(int(ia.bytes), dtype=torch.uint8, device="cuda")
        oc = torch.empty(int(ic.bytes), dtype=torch.uint8, device="cuda")
        with VoxelizerBatch() as b:
            b.add(a, 1, 32, oa)
            with pytest.raises(Exception):
                b.add(c, 1, 32, oc)
