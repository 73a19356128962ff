"""Continuous-batching voxelization service on one GPU.

Requests (a mesh plus the arguments of one ``voxelizeToNodes`` call) are
taken in by a pool of ingest threads (mesh checks, bounding box, upload to
the device, grid plan) and queued as they become ready.  Worker lanes, each
with its own CUDA stream and ``vxb_batch``, repeatedly take every waiting
request that fits the free device-memory budget and run them as one batch
(one sequence of launches for all of them, vxb_batch_run).  While one lane's batch is on the GPU the next
lane forms and launches the following batch from the requests that arrived
meanwhile, so work of different batches overlaps on the device.  Results
stay resident in device memory until the caller fetches or releases them;
their bytes count against the budget until then.

Each result is identical to a single ``vxb_voxelize_to_device`` call on the
same mesh and arguments: a batch runs the same kernels on the same inputs,
and no kernel's output depends on the other meshes of its batch.
"""

from __future__ import annotations

import threading
import time
from collections import deque

import numpy as np

from .api import DEFAULT_MAT, DEFAULT_VOX, LONG, Voxelizer, VoxelizerBatch


class Request:
    """One voxelization job; ``wait()`` blocks until its result is ready."""

    def __init__(self, mesh_v, mesh_i, mats, n_mats, size, node_type, vox, mat, t_submit=None):
        self.t_submit = time.perf_counter() if t_submit is None else t_submit
        self.voxelizer = Voxelizer(mesh_v, mesh_i, mats, n_mats, node_type=node_type)
        self.size = size
        self.vox = vox
        self.mat = mat
        self.info = self.voxelizer.plan(1, size, vox, mat)
        n_t = int(np.asarray(mesh_i).size // 3)
        n_v = int(np.asarray(mesh_v).size // 3)
        words = int(self.info.count) // 8 + 64
        # Output plus the resident mesh plus this request's share of the
        # batch pipeline's buffers (bit grids, ranks, work lists, records).
        self.bytes = int(self.info.bytes) + 13 * n_t + 12 * n_v + 16 * words + 200 * n_t
        self.t_done = None
        self.out = None
        self.error = None
        self._event = threading.Event()

    @property
    def latency(self):
        return None if self.t_done is None else self.t_done - self.t_submit

    def wait(self, timeout=None):
        if not self._event.wait(timeout):
            raise TimeoutError("request not finished")
        if self.error:
            raise self.error
        return self.out


class Pending:
    """A submitted request before ingestion; ``wait()`` returns the result."""

    def __init__(self, args):
        self.args = args
        self.t_submit = time.perf_counter()
        self.request = None
        self.error = None
        self._ready = threading.Event()

    def _resolve(self):
        self._ready.wait()
        if self.error:
            raise self.error
        return self.request

    def wait(self, timeout=None):
        return self._resolve().wait(timeout)

    @property
    def t_done(self):
        return self._resolve().t_done

    @property
    def latency(self):
        r = self._resolve()
        return None if r.t_done is None else r.t_done - self.t_submit


class VoxelServer:
    """``submit`` returns a Pending handle; ``fetch`` returns its device
    result and releases its budget; ``close`` drains and stops the threads."""

    def __init__(self, budget_bytes=160 << 30, lanes=2, max_batch=256, device=0, ingest_threads=3):
        import torch

        self.torch = torch
        self.device = device
        self.budget = int(budget_bytes)
        self.max_batch = int(max_batch)
        self._used = 0
        self._queue: deque[Request] = deque()
        self._cv = threading.Condition()
        self._stop = False
        self.batches = 0
        self.batched_requests = 0
        self._incoming: deque[Pending] = deque()
        self._in_cv = threading.Condition()
        self._ingest = [threading.Thread(target=self._ingest_loop, daemon=True) for _ in range(ingest_threads)]
        self._lanes = [threading.Thread(target=self._lane, args=(k,), daemon=True) for k in range(lanes)]
        for t in self._ingest + self._lanes:
            t.start()

    # -- client side --
    def submit(self, vertices, indices, materials=None, n_materials=None, size=256, node_type=LONG,
               vox=DEFAULT_VOX, mat=DEFAULT_MAT):
        """Queues one job; the arrays must stay unchanged until its ingestion
        (the Pending's wait() returning, or fetch)."""
        p = Pending((vertices, indices, materials, n_materials, size, node_type, vox, mat))
        with self._in_cv:
            self._incoming.append(p)
            self._in_cv.notify()
        return p

    def fetch(self, req, host=False):
        """The node grid (a device tensor, or a numpy array with host=True);
        releases the request's device memory budget."""
        out = req.wait()
        res = out.cpu().numpy() if host else out
        self.release(req)
        return res

    def release(self, req):
        if isinstance(req, Pending):
            req = req._resolve()
        with self._cv:
            if req.out is not None:
                req.out = None
                self._used -= req.bytes
                self._cv.notify_all()
            req.voxelizer.close()

    def close(self):
        with self._in_cv:
            self._stop = True
            self._in_cv.notify_all()
        for t in self._ingest:
            t.join()
        with self._cv:
            self._cv.notify_all()
        for t in self._lanes:
            t.join()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- ingestion --
    def _ingest_loop(self):
        torch = self.torch
        torch.cuda.set_device(self.device)
        while True:
            with self._in_cv:
                while not self._incoming and not self._stop:
                    self._in_cv.wait(0.05)
                if not self._incoming:
                    return
                p = self._incoming.popleft()
            try:
                req = Request(*p.args, t_submit=p.t_submit)
                if req.bytes > self.budget:
                    req.voxelizer.close()
                    raise ValueError(f"request needs {req.bytes} bytes, more than the whole budget ({self.budget})")
                with self._cv:
                    self._queue.append(req)
                    self._cv.notify()
                p.request = req
            except Exception as e:  # noqa: BLE001 - reported to the caller through the Pending
                p.error = e
            p._ready.set()

    # -- lanes --
    def _take(self):
        """Every waiting request that fits the free budget (FIFO; a request
        that does not fit waits for memory)."""
        with self._cv:
            while True:
                if self._stop and not self._queue and not any(t.is_alive() for t in self._ingest):
                    return None
                batch = []
                while self._queue and len(batch) < self.max_batch:
                    r = self._queue[0]
                    if self._used + r.bytes > self.budget:
                        break
                    self._queue.popleft()
                    self._used += r.bytes
                    batch.append(r)
                if batch:
                    return batch
                self._cv.wait(0.05)

    def _lane(self, k):
        torch = self.torch
        torch.cuda.set_device(self.device)
        stream = torch.cuda.Stream()
        vb = VoxelizerBatch(device=self.device)
        while True:
            reqs = self._take()
            if reqs is None:
                break
            try:
                vb.clear()
                with torch.cuda.stream(stream):
                    outs = [torch.empty(int(r.info.bytes), dtype=torch.uint8, device="cuda") for r in reqs]
                for r, o in zip(reqs, outs):
                    vb.add(r.voxelizer, 1, r.size, o, r.vox, r.mat)
                vb.run(stream=stream.cuda_stream)
                now = time.perf_counter()
                for r, o in zip(reqs, outs):
                    r.out = o
                    r.t_done = now
                    r._event.set()
                with self._cv:
                    self.batches += 1
                    self.batched_requests += len(reqs)
            except Exception as e:  # noqa: BLE001 - reported to every request of the batch
                with self._cv:
                    for r in reqs:
                        self._used -= r.bytes
                for r in reqs:
                    r.error = e
                    r.t_done = time.perf_counter()
                    r._event.set()
        vb.close()
