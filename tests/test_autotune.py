"""Launch-shape autotuner (vxb_set_autotune): shapes change only how kernels
spread their work, so every trial and every settled shape must give the
same output; settled shapes go to a JSON cache that a later process can use
unchanged (mode 2)."""

import json

import numpy as np
import pytest

from voxelizer_b200 import _lib
from voxelizer_b200.api import LONG, Voxelizer
from voxelizer_b200.scenes import Mesh, icosphere, torus


@pytest.fixture(autouse=True)
def _tuner_off():
    yield
    _lib.set_autotune(0)


def test_modes_and_cache_file(tmp_path):
    path = tmp_path / "shapes.json"
    good = {"surf_blocks_per_sm": 16, "surf_batch": 8, "merge_blocks_per_sm": 4, "emit_blocks_per_sm": 8,
            "toggle_blocks_per_sm": 6, "surf_queue": 1, "toggle_queue": 1, "surf_merge": 1}
    bad_shape = dict(good, surf_blocks_per_sm=7)
    bad_merge = dict(good, surf_merge=2)
    old_format = {k: v for k, v in good.items() if k != "surf_merge"}
    path.write_text("{\n" + ",\n".join(f'  "{k}": {json.dumps(v)}' for k, v in (
        ("t12-w17-k1-m1", good), ("t13-w17-k1-m1", bad_shape), ("t14-w17-k1-m1", bad_merge),
        ("t15-w17-k1-m1", old_format))) + "\n}\n")
    _lib.set_autotune(2, str(path))
    n, text = _lib.autotune_state()
    # Entries naming a value that is not a candidate, or lacking a field of
    # the current format, are skipped.
    assert n == 1
    assert json.loads(text) == {"t12-w17-k1-m1": good}
    with pytest.raises(_lib.VxbError, match="EINVAL"):
        _lib.set_autotune(3)
    _lib.set_autotune(0)
    assert _lib.autotune_state()[0] == 0


@pytest.mark.gpu
def test_tuning_keeps_results_and_settles(tmp_path):
    v, f = torus(96, 48, 0.6, 0.25)
    m = Mesh(v, f, (1 + np.arange(f.shape[0]) % 5).astype(np.uint8), 6)
    path = tmp_path / "shapes.json"
    with Voxelizer(m.vertices, m.indices, m.materials, m.n_materials, node_type=LONG) as vx:
        want, _ = vx.voxelizeToNodesToRAM(160)
        wbits, _ = vx.voxelizeToRAM(160)
        _lib.set_autotune(1, str(path))
        # 3 shape candidates x 3 samples, then (node grids with materials)
        # 2 material-key strategies x 3 samples settle a bucket.
        for _ in range(16):
            got, _ = vx.voxelizeToNodesToRAM(160)
            assert np.array_equal(got, want)
            bits, _ = vx.voxelizeToRAM(160)
            assert np.array_equal(bits, wbits)
        n, text = _lib.autotune_state()
        assert n >= 2   # the node bucket and the bit-array bucket
        assert json.loads(path.read_text()) == json.loads(text)
        # A later process reads the cache without tuning (mode 2).
        _lib.set_autotune(2, str(path))
        assert _lib.autotune_state()[0] == n
        got, _ = vx.voxelizeToNodesToRAM(160)
        assert np.array_equal(got, want)
        # Both material-key strategies, forced through the cache, give the
        # same node grid.
        shapes = json.loads(text)
        for merge in (0, 1):
            path.write_text("{\n" + ",\n".join(f'  "{k}": {json.dumps(dict(s, surf_merge=merge))}'
                                                for k, s in shapes.items()) + "\n}\n")
            _lib.set_autotune(2, str(path))
            for nodes in (True, False):
                got, _ = vx.voxelizeToNodesToRAM(160) if nodes else vx.voxelizeToRAM(160)
                assert np.array_equal(got, want if nodes else wbits), merge
