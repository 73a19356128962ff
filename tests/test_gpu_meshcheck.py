"""vxb_create checks the mesh on the device when it has one (largest index,
first out-of-range index, bounding box).  The results must equal the host
scan's (device -1 keeps everything on the host): the same error for the
same bad index, and the same box, including the scan's order rules (the
first of equal extremes wins, so -0 and +0 keep their first sign; NaN
coordinates after vertex 0 are never taken; a NaN in vertex 0 stays)."""

import numpy as np
import pytest

from voxelizer_b200 import _lib
from voxelizer_b200.api import Voxelizer

pytestmark = pytest.mark.gpu


def host_scan(v):
    """The sequential scan the host runs (boundingBox in vxb_plan.h)."""
    mn = [float(v[0, a]) for a in range(3)]
    mx = list(mn)
    for p in v[1:]:
        for a in range(3):
            if p[a] > mx[a]:
                mx[a] = float(p[a])
            if p[a] < mn[a]:
                mn[a] = float(p[a])
    return mn, mx


def infos(v, f, size=64):
    out = []
    for dev in (0, -1):
        with Voxelizer(v, f, device=dev) as vx:
            out.append(vx.plan(1, size))
    return out


def same_bits(a, b):
    return np.array(a, np.float64).view(np.uint64).tolist() == np.array(b, np.float64).view(np.uint64).tolist()


def test_box_matches_host_scan_on_random_meshes():
    rng = np.random.default_rng(7)
    for n in (3, 4, 1000, 250_001):
        v = rng.normal(size=(n, 3)).astype(np.float32)
        v[rng.integers(0, n, size=n // 10)] = v[0]          # repeated extremes
        f = rng.integers(0, n, size=(max(n // 2, 1), 3)).astype(np.uint32)
        dev, host = infos(v, f)
        mn, mx = host_scan(v)
        assert list(dev.min_vertex) == list(host.min_vertex) == mn
        assert list(dev.max_vertex) == list(host.max_vertex)
        assert dev.dims == host.dims and dev.voxel_length == host.voxel_length


def test_box_order_rules():
    # Zeros of both signs at the extremes, NaNs after vertex 0.
    v = np.array([[1, 1, 1], [-0.0, 2, 0.0], [0.0, np.nan, -0.0], [3, -0.0, 5], [0.0, 0.0, -1]], np.float32)
    f = np.array([[0, 1, 2], [2, 3, 4]], np.uint32)
    dev, host = infos(v, f)
    mn, mx = host_scan(v)
    assert same_bits(list(dev.min_vertex), mn) and same_bits(list(host.min_vertex), mn)
    assert same_bits(list(dev.max_vertex), list(host.max_vertex))


def test_bad_index_error_matches_host():
    rng = np.random.default_rng(3)
    v = rng.normal(size=(500, 3)).astype(np.float32)
    f = rng.integers(0, 500, size=(3000, 3)).astype(np.uint32)
    f[1234, 2] = 500
    f[2000, 0] = 9999
    msgs = []
    for dev in (0, -1):
        with pytest.raises(_lib.VxbError) as e:
            Voxelizer(v, f, device=dev)
        assert e.value.status == -1
        msgs.append(str(e.value))
    assert msgs[0] == msgs[1]
    assert "index 500 of triangle 1234 is out of range" in msgs[0]
