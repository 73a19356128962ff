"""The contraction model against the reference's own output at exact ties.

tests/golden/fma_probe_nt{0..4}.npz hold, per node type, the surface nodes
that the reference's CUDA kernels (built from src/voxelizer.cu for sm_100a)
produced for 60 scenes of isolated triangles whose vertices sit on voxel
centres, cell faces and cell corners (tests/golden/make_fma_probe.py).  At
those ties the conservative triangle/box tests (src/voxelizer.cu:2633-2942,
3306-4119) decide by the last bit, so every site of the contraction model
(voxelizer_b200/csrc/vxb_sites.inc) is exercised: the CPU test checks the
oracle, which evaluates the same table, and the GPU test the CUDA path.
"""

import os

import numpy as np
import pytest

import make_fma_probe as P
import oracle as O

GOLD = os.path.dirname(os.path.abspath(__file__)) + "/golden"
NODE_TYPES = [0, 1, 2, 3, 4]
FCC = {3, 4}


def _gold(nt):
    return np.load(os.path.join(GOLD, f"fma_probe_nt{nt}.npz"))


def _oracle_surface(m, nt, d, n, model=None):
    pred = np.zeros(n, bool)
    for g in ([1, 2, 3, 4] if nt in FCC else [0]):
        pred[O.surface_hits(m, nt, float(d), g, fma_model=model)[:, 1]] = True
    return pred


def _mismatches(nt, model=None):
    z = _gold(nt)
    bad = 0
    for s in range(P.SCENES):
        m, d = P.scene(s)
        dims = tuple(int(x) for x in z[f"s{s}_dims"])
        n = int(np.prod(dims))
        want = np.zeros(n, bool)
        want[z[f"s{s}_idx"]] = True
        bad += int(np.count_nonzero(_oracle_surface(m, nt, d, n, model) != want))
    return bad


@pytest.mark.parametrize("nt", NODE_TYPES)
def test_oracle_matches_reference_probe(nt):
    """Every surface node of every probe scene, per node type."""
    assert _mismatches(nt) == 0


def test_probe_discriminates_the_model():
    """The probe is sensitive to the fitted forms: the LongNode model with the
    ShortNode depth-loop prolog form, or without the unrolled prologs, no
    longer matches the LongNode probe."""
    for change in ({"OT_3DXP_ZX": 21}, {"UNR_2D": 0}, {"UNR_3DL": 0}, {"DT_3DX": 1}):
        model = dict(O.PINNED_FMA)
        model.update(change)
        assert _mismatches(1, model) > 0, change


@pytest.mark.gpu
@pytest.mark.parametrize("nt", NODE_TYPES)
def test_cuda_matches_reference_probe(nt):
    """The CUDA path through the C ABI, node grid with materials, against
    the reference's surface nodes."""
    import torch

    from voxelizer_b200.api import Voxelizer

    assert torch.cuda.is_available()
    z = _gold(nt)
    for s in range(P.SCENES):
        m, d = P.scene(s)
        with Voxelizer(m.vertices, m.indices, node_type=nt) as v:
            v.setMaterials(m.materials, m.n_materials)
            out, info = v.voxelizeToNodesToRAM(float(d))
        assert tuple(info.dims) == tuple(int(x) for x in z[f"s{s}_dims"])
        got = P.surface_nodes(nt, out)
        want = z[f"s{s}_idx"]
        assert np.array_equal(got, want), f"scene {s}: {np.setxor1d(got, want).size} surface nodes differ"
