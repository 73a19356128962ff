"""The continuous-batching server: every result equals the single call on the
same mesh and arguments, whatever the batch it ran in; a small memory budget
delays requests but completes them all."""

import threading

import numpy as np
import pytest

import cases as C
from voxelizer_b200 import scenes
from voxelizer_b200.api import DEFAULT_MAT, DEFAULT_VOX, LONG, Voxelizer
from voxelizer_b200.serve import Request, VoxelServer

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _jobs():
    jobs = []
    for k, (lvl, r) in enumerate(((2, 0.3), (3, 0.4), (4, 0.45), (3, 0.2), (2, 0.5), (4, 0.35))):
        v, f = scenes.icosphere(lvl, r, (0.1 * k, 0.0, 0.2))
        m = (1 + np.arange(f.shape[0]) % (k + 2)).astype(np.uint8)
        jobs.append((scenes.Mesh(v, f, m, k + 3, f"ico{lvl}_{k}"), 24 + 13 * k))
    jobs.append((C.mesh("torus"), 90))
    jobs.append((C.mesh("room_lite"), 100))
    return jobs


def _alone(mesh, size):
    with Voxelizer(mesh.vertices, mesh.indices, mesh.materials, mesh.n_materials, node_type=LONG) as v:
        info = v.plan(1, size)
        out = torch.empty(int(info.bytes), dtype=torch.uint8, device="cuda")
        v.voxelize_device(1, size, out)
        torch.cuda.synchronize()
        return out


@pytest.mark.parametrize("lanes", [1, 2])
def test_served_results_equal_single_calls(lanes):
    jobs = _jobs() * 3
    ref = [_alone(m, s) for m, s in jobs]
    pairs = []
    lock = threading.Lock()
    with VoxelServer(lanes=lanes) as srv:
        def submit_all(idx):
            for j in idx:
                m, s = jobs[j]
                r = srv.submit(m.vertices, m.indices, m.materials, m.n_materials, size=s)
                with lock:
                    pairs.append((r, j))

        # Three clients submitting at once: requests land in shared batches.
        ths = [threading.Thread(target=submit_all, args=(range(i, len(jobs), 3),)) for i in range(3)]
        for t in ths:
            t.start()
        for t in ths:
            t.join()
        assert len(pairs) == len(jobs)
        for r, j in pairs:
            assert torch.equal(srv.fetch(r), ref[j]), f"job {j} differs from its single call"
        assert 1 <= srv.batches <= len(jobs)


def test_served_small_budget_completes():
    jobs = _jobs()
    ref = [_alone(m, s) for m, s in jobs]
    need = []
    for m, s in jobs:
        r = Request(m.vertices, m.indices, m.materials, m.n_materials, s, LONG, DEFAULT_VOX, DEFAULT_MAT)
        need.append(r.bytes)
        r.voxelizer.close()
    # Room for about two requests at a time: the rest wait for memory.
    with VoxelServer(lanes=2, budget_bytes=2 * max(need)) as srv:
        reqs = [srv.submit(m.vertices, m.indices, m.materials, m.n_materials, size=s) for m, s in jobs]
        for r, want in zip(reqs, ref):
            assert torch.equal(srv.fetch(r), want)
        assert srv.batches >= 2
