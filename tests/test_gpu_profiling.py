"""Stage timing (vxb_set_profiling, vxb_stage_times, vxb_stage_timeline):
events change no result, every stage of a node grid with materials is
timed, and the timeline shows the order the streams impose: the surface
work inside the surface stage, emission after both pruning and the
material merge.  The serial mode runs the stages one after another."""

import math

import numpy as np
import pytest

from voxelizer_b200.api import LONG, Voxelizer
from voxelizer_b200.scenes import Mesh, torus


@pytest.mark.gpu
def test_stage_times_and_timeline():
    v, f = torus(96, 48, 0.6, 0.25)
    m = Mesh(v, f, (1 + np.arange(f.shape[0]) % 5).astype(np.uint8), 6)
    with Voxelizer(m.vertices, m.indices, m.materials, m.n_materials, node_type=LONG) as vx:
        want, _ = vx.voxelizeToNodesToRAM(160)
        assert all(math.isnan(a) for a, _ in vx.stage_timeline().values())
        vx.set_profiling(True)
        got, _ = vx.voxelizeToNodesToRAM(160)
        assert np.array_equal(got, want)
        ms = vx.stage_times()
        tl = vx.stage_timeline()
        vx.set_profiling(False)
    assert all(ms[k] >= 0.0 for k in Voxelizer.STAGES), ms
    assert tl["solid"][0] == 0.0
    for k, (a, b) in tl.items():
        assert a <= b, (k, a, b)
        assert abs((b - a) - ms[k]) < 1e-2, (k, b - a, ms[k])
    eps = 1e-3
    assert tl["surface"][0] - eps <= tl["surface_work"][0] and tl["surface_work"][1] <= tl["surface"][1] + eps
    assert tl["emit"][0] + eps >= tl["prune"][1]
    assert tl["emit"][0] + eps >= tl["merge"][1]
    assert tl["prune"][0] + eps >= tl["solid"][1]


@pytest.mark.gpu
def test_serial_profiling_keeps_results_and_orders_the_stages():
    v, f = torus(96, 48, 0.6, 0.25)
    m = Mesh(v, f, (1 + np.arange(f.shape[0]) % 5).astype(np.uint8), 6)
    with Voxelizer(m.vertices, m.indices, m.materials, m.n_materials, node_type=LONG) as vx:
        want, _ = vx.voxelizeToNodesToRAM(160)
        vx.set_profiling(True, serial=True)
        got, _ = vx.voxelizeToNodesToRAM(160)
        tl = vx.stage_timeline()
        vx.set_profiling(False)
        assert np.array_equal(got, want)
    eps = 1e-3
    # The surface pass (with its merge) runs first, then the solid pass,
    # pruning and emission, none beside another.
    assert tl["surface"][1] <= eps and tl["merge"][1] <= eps
    assert tl["prune"][0] + eps >= tl["solid"][1]
    assert tl["emit"][0] + eps >= tl["prune"][1]
