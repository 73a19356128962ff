"""Benchmark of the mesh -> node-grid path.

Workload (one step): the room scene -- an inward 10 x 7.5 x 5 box shell plus
200 rotated icospheres / tori, 1,049,868 float32 triangles, 17 materials --
voxelized with Voxelizer<LongNode>::voxelizeToNodesToRAM(1024) semantics:
solid + surface voxelization, split-ordered pruning and node emission into a
1088 x 771 x 515 LongNode grid (432,006,720 nodes, 864 MB).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

value: Gvoxels/s of node grid, device resident (mesh already on the GPU,
  output in HBM), timed with CUDA events on the launching stream; the L2 is
  flushed (256 MB write) before every timed step.
e2e: the same metric through the reference-facing C ABI with host buffers:
  each step constructs the voxelizer from pinned host arrays, uploads the
  mesh, voxelizes and copies the node grid back into pinned host memory.
--impl reference: the reference's own implementation of the path through
  its public API (Voxelizer<LongNode>::voxelizeToNodesToRAM, src/host_side.cpp
  with its CUDA kernels src/voxelizer.cu), built from its sources into
  oracle/_ref/ and run on cuda:0 with host arrays in and out, on the full
  workload.  It has no CPU code; where that library or a GPU is missing, the
  CPU restatement (oracle/) runs on all host cores on a bounded sample.
Multi-GPU: replicas only (the path does not shard); under torchrun every
rank voxelizes its own copy and value sums the voxels of all ranks over the
slowest rank's time.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "node-grid voxelization throughput (Gvoxels/s), bit-exact vs reference"
UNIT = "Gvoxels/s"
WORKLOAD = "room scene, 1,049,868 triangles, 17 materials, LongNode, maxDimension 1024 -> 1088x771x515 nodes"
# The same config dict in both arms: the workload and how the L2 is kept out
# of the timing (every step writes an 864 MB node grid).
L2_NOTE = ("each step writes an 864 MB node grid (L2 126 MB); the device-resident timing also writes 256 MB "
           "to flush the L2 before every timed step")
CONFIG = {"workload": WORKLOAD, "l2": L2_NOTE}
MAX_DIM = 1024
CPU_SAMPLE_DIM = 384


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            p = json.load(fh)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(key):
    """Per-launch DRAM bytes (read + write) of a kernel from the committed ncu
    summary profiles/ncu_traffic.txt, or None."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    try:
        with open(path) as fh:
            for line in fh:
                k, _, v = line.partition("=")
                if k.strip() == key:
                    return float(v)
    except OSError:
        pass
    return None


class ClockSampler:
    """SM clock and throttle-reason samples while the timed region runs:
    NVML polled every 5 ms from a thread (reads only), else nvidia-smi at its
    shortest period."""

    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20, "sw_power_cap": 0x4}

    def __init__(self, index, period_s=0.005):
        self.index = index
        self.period = period_s
        self.samples = []   # (sm_mhz, max_mhz, reasons set)
        self._stop = threading.Event()
        self._proc = None
        self._thread = None
        self._nvml = None

    def __enter__(self):
        try:
            import pynvml

            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            mx = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
            self._nvml = pynvml

            def poll():
                while not self._stop.is_set():
                    sm = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
                    bits = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                    self.samples.append((float(sm), float(mx),
                                         {n for n, b in self.REASONS.items() if bits & b}))
                    self._stop.wait(self.period)

            self._thread = threading.Thread(target=poll, daemon=True)
            self._thread.start()
            return self
        except Exception:
            self._nvml = None
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self._proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                           "-i", str(self.index), "-lms", "20"], stdout=subprocess.PIPE,
                                          stderr=subprocess.DEVNULL, text=True)
            self._thread = threading.Thread(target=self._read, daemon=True)
            self._thread.start()
        except OSError:
            self._proc = None
        return self

    def _read(self):
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self._proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 8 and parts[1].replace(".", "").isdigit():
                self.samples.append((float(parts[1]), float(parts[2]),
                                     {names[i] for i in range(4) if parts[4 + i] == "Active"}))

    def __exit__(self, *a):
        self._stop.set()
        if self._proc:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self._proc.kill()
        if self._thread:
            self._thread.join(timeout=5)
        if self._nvml:
            try:
                self._nvml.nvmlShutdown()
            except Exception:
                pass

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = sorted(s[0] for s in self.samples)
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": max(s[1] for s in self.samples),
                "reasons": sorted(set().union(*(s[2] for s in self.samples))), "samples": len(self.samples),
                "source": "nvml" if self._nvml else "nvidia-smi"}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libvoxref.so")


def _reference_cuda():
    """The reference's own CUDA kernels (src/voxelizer.cu compiled from its
    sources by oracle/Makefile) with the driver of oracle/ref_driver.cu, or
    None where that library or a GPU is missing."""
    if not os.path.exists(REF_LIB):
        return None
    try:
        import torch

        if not torch.cuda.is_available():
            return None
    except ImportError:
        return None
    import ctypes

    lib = ctypes.CDLL(REF_LIB)
    f = lib.ref_voxelize
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint32, ctypes.c_double,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p,
                  ctypes.c_uint32, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_uint64,
                  ctypes.c_void_p, ctypes.c_void_p]
    lib.ref_last_error.restype = ctypes.c_char_p
    return f, lib


def max_over_ranks(x, dist):
    """The largest x over the ranks of the process group (a job's time is
    its slowest replica's).  NCCL reduces a device tensor, gloo a host one."""
    import torch

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(units_per_replica, world, ms):
    """Whole-job units per second: every replica processes the same units
    in (at most) `ms` milliseconds."""
    return units_per_replica * world / (ms * 1e-3)


def run_reference_cuda(args, world, ref):
    """Full workload through the reference's CUDA path on cuda:0: host arrays
    in, node grid back in host memory, wall clock per call (the reference's
    voxelizeToNodesToRAM allocates, uploads, computes and copies back inside
    the call)."""
    import ctypes

    from voxelizer_b200 import scenes

    f, lib = ref
    mesh = scenes.room_scene()
    vox = np.array([1024, 512, 512], dtype=np.uint32)
    mat = np.array([512, 512, 512], dtype=np.uint32)
    dims = np.zeros(3, dtype=np.uint32)
    ms = ctypes.c_double(0.0)
    v = np.ascontiguousarray(mesh.vertices.reshape(-1))
    i = np.ascontiguousarray(mesh.indices.reshape(-1))
    m = np.ascontiguousarray(mesh.materials)
    args_common = (1, 1, 1, 0, MAX_DIM, 0.0, vox.ctypes.data, mat.ctypes.data, v.ctypes.data, mesh.n_vertices,
                   i.ctypes.data, mesh.n_triangles, m.ctypes.data, mesh.n_materials)
    rc = f(*args_common, None, 0, dims.ctypes.data, None)
    if rc != 0:
        raise RuntimeError(f"reference plan failed ({rc}): {lib.ref_last_error().decode()}")
    n_nodes = int(dims[0]) * int(dims[1]) * int(dims[2])
    out = np.empty(n_nodes, dtype=np.uint16)
    times = []
    for k in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        rc = f(*args_common, out.ctypes.data, out.nbytes, dims.ctypes.data, ctypes.byref(ms))
        dt = time.perf_counter() - t0
        if rc != 0:
            raise RuntimeError(f"reference run failed ({rc}): {lib.ref_last_error().decode()}")
        if k >= args.warmup:
            times.append(dt)
    t = sum(times)
    value = n_nodes * len(times) / t / 1e9
    sample = (f"full workload, {int(dims[0])}x{int(dims[1])}x{int(dims[2])} nodes per step: the reference's own "
              f"CUDA kernels (src/voxelizer.cu built from its sources for sm_100a) on cuda:0, host arrays in and "
              f"out, wall clock per call")
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 6), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * t / len(times), 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32+u32",
            "data": "synthetic (seeded room scene)", "device": "cuda:0",
            "config": dict(CONFIG), "sample": sample,
            "cpu_baseline": {"value": round(value, 6), "unit": UNIT, "cores": 1, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": round(value, 6), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_reference_api(args, world):
    """Full workload through the reference's own public API on cuda:0:
    vox::Voxelizer<LongNode>::voxelizeToNodesToRAM(1024) of its
    src/host_side.cpp and src/voxelizer.cu, built from its sources
    (oracle/_ref/libvoxhost.so).  Host arrays in, node grid back in host
    memory, wall clock per call (the call allocates, uploads, computes and
    copies back)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_host as RH
    from voxelizer_b200 import scenes

    mesh = scenes.room_scene()
    out, dims, _ = RH.voxelize(mesh, 1, 1, MAX_DIM)
    n_nodes = dims[0] * dims[1] * dims[2]
    times = []
    for k in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        RH.voxelize(mesh, 1, 1, MAX_DIM, out=out)
        dt = time.perf_counter() - t0
        if k >= args.warmup:
            times.append(dt)
    t = sum(times)
    value = n_nodes * len(times) / t / 1e9
    sample = (f"full workload, {dims[0]}x{dims[1]}x{dims[2]} nodes per step: the reference's own public API "
              f"(Voxelizer<LongNode>::voxelizeToNodesToRAM of src/host_side.cpp with src/voxelizer.cu, built from "
              f"its sources for sm_100a) on cuda:0, host arrays in and out, wall clock per call")
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 6), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * t / len(times), 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32+u32",
            "data": "synthetic (seeded room scene)", "device": "cuda:0",
            "config": dict(CONFIG), "sample": sample,
            "cpu_baseline": {"value": round(value, 6), "unit": UNIT, "cores": 1, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": round(value, 6), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_reference(args, world, rank):
    """The reference's implementation of the path: its own public API where
    it was built from its sources, else its kernels behind the restated
    host flow of oracle/ref_driver.cu, else its CPU restatement (oracle/) on
    all host cores."""
    if rank != 0:
        return
    if os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libvoxhost.so")) and _reference_cuda() is not None:
        run_reference_api(args, world)
        return
    ref = _reference_cuda()
    if ref is not None:
        run_reference_cuda(args, world, ref)
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from voxelizer_b200 import scenes

    mesh = scenes.room_scene()
    cores = os.cpu_count() or 1
    times = []
    info = None
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        out, info, _ = O.voxelize(mesh, 1, 1, 1, CPU_SAMPLE_DIM, threads=cores)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            times.append(dt)
        del out
    n = info.dims[0] * info.dims[1] * info.dims[2]
    t = sum(times)
    value = n * len(times) / t / 1e9
    sample = (f"room scene (1,049,868 triangles, 17 materials), LongNode, maxDimension {CPU_SAMPLE_DIM} -> "
              f"{info.dims[0]}x{info.dims[1]}x{info.dims[2]} nodes per step (full path)")
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 6), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * t / len(times), 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32+u32",
            "data": "synthetic (seeded room scene)",
            "config": dict(CONFIG), "sample": sample,
            "cpu_baseline": {"value": round(value, 6), "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": sample},
            "e2e": {"value": round(value, 6), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def cpu_baseline(mesh):
    """One run of the CPU restatement (oracle/) of the reference's kernels on
    the full workload, all host cores."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    out, info, _ = O.voxelize(mesh, 1, 1, 1, MAX_DIM, threads=cores)
    dt = time.perf_counter() - t0
    n = info.dims[0] * info.dims[1] * info.dims[2]
    del out
    return {"value": round(n / dt / 1e9, 6), "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"the full workload ({info.dims[0]}x{info.dims[1]}x{info.dims[2]} nodes), one run of the "
                      f"whole path, {dt:.1f} s on {cores} threads"}


def profile_run(args):
    """The workload's launches and nothing else, for a profiler to capture:
    the room scene at maxDimension --profile-run, or with --workload batched
    the 256-mesh mix as one batch (without graph capture)."""
    import torch

    from voxelizer_b200 import scenes
    from voxelizer_b200.api import LONG, Voxelizer, VoxelizerBatch

    if args.workload == "batched":
        mix = scenes.batch_mix(args.batch_meshes, seed=0)
        keep = []
        with VoxelizerBatch() as b:
            for mesh, md in mix:
                v = Voxelizer(mesh.vertices, mesh.indices, mesh.materials, mesh.n_materials, node_type=LONG)
                o = torch.empty(int(v.plan(1, md).bytes), dtype=torch.uint8, device="cuda")
                keep.append((v, o))
                b.add(v, 1, md, o)
            for _ in range(args.steps):
                b.run()
            torch.cuda.synchronize()
            print(f"profile run: {args.steps} x batch of {len(mix)}, {b.last_launch_count()} launches each", flush=True)
        return
    mesh = scenes.room_scene()
    with Voxelizer(mesh.vertices, mesh.indices, mesh.materials, mesh.n_materials, node_type=LONG) as vx:
        info = vx.plan(1, args.profile_run)
        out = torch.empty(int(info.bytes), dtype=torch.uint8, device="cuda")
        for _ in range(args.steps):
            vx.voxelize_device(1, args.profile_run, out)
        torch.cuda.synchronize()
        print(f"profile run: {args.steps} x {info.dims}, {vx.last_launch_count()} launches each", flush=True)


BATCH_METRIC = "batched meshes/s (256-mesh mix, LongNode with materials), bit-exact vs per-mesh calls"


def run_batched(args, world, rank, local):
    """The 256-mesh mix: one batch (graph replay) against a loop of plain
    per-mesh calls, same outputs.  Each rank runs its own copy (replicas)."""
    line = batched_line(args, world, local, args.steps, args.warmup)
    if rank == 0:
        print(json.dumps(line), flush=True)


def batched_line(args, world, local, steps, warmup):
    """The batched workload's result line (see run_batched)."""
    import torch

    from voxelizer_b200 import scenes
    from voxelizer_b200.api import LONG, Voxelizer, VoxelizerBatch

    torch.cuda.set_device(local)
    mix = scenes.batch_mix(args.batch_meshes, seed=0)
    vxs, outs_loop, outs_batch, infos = [], [], [], []
    for mesh, md in mix:
        v = Voxelizer(mesh.vertices, mesh.indices, mesh.materials, mesh.n_materials, node_type=LONG, device=local)
        info = v.plan(1, md)
        vxs.append(v)
        infos.append(info)
        outs_loop.append(torch.empty(int(info.bytes), dtype=torch.uint8, device="cuda"))
        outs_batch.append(torch.empty(int(info.bytes), dtype=torch.uint8, device="cuda"))
    n_nodes = sum(int(i.count) for i in infos)
    n_tris = sum(int(m.n_triangles) for m, _ in mix)
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream

    def loop():
        for (mesh, md), v, o in zip(mix, vxs, outs_loop):
            v.voxelize_device(1, md, o, stream=sh)

    batch = VoxelizerBatch(device=local)
    for (mesh, md), v, o in zip(mix, vxs, outs_batch):
        batch.add(v, 1, md, o)

    def timed(fn, steps):
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        torch.cuda.synchronize()
        for a, b in evs:
            a.record(stream)
            fn()
            b.record(stream)
        torch.cuda.synchronize()
        return sum(a.elapsed_time(b) for a, b in evs) / steps

    def tune_calls():
        loop()
        batch.run(stream=sh, graph=False)
        stream.synchronize()

    tuned = autotune(args, tune_calls)
    for _ in range(warmup):
        loop()
        batch.run(stream=sh, graph=True)
    launches = batch.last_launch_count()
    t_loop = timed(loop, max(1, steps // 2))
    with ClockSampler(local) as clk:
        t_batch = timed(lambda: batch.run(stream=sh, graph=True), steps)
    same = all(torch.equal(a, b) for a, b in zip(outs_loop, outs_batch))
    batch.close()
    for v in vxs:
        v.close()
    value = args.batch_meshes * world / (t_batch * 1e-3)
    line = {"metric": BATCH_METRIC, "value": round(value, 2), "unit": "meshes/s", "n_gpus": world,
            "steps": steps, "warmup": warmup, "ms_per_step": round(t_batch, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32+u32",
            "data": f"synthetic (seeded {args.batch_meshes}-mesh mix: icospheres/tori, 500-500k triangles, "
                    "maxDimension 32-512, 1-16 materials)",
            "config": {"workload": f"{args.batch_meshes} meshes, {n_tris:,} triangles, {n_nodes:,} nodes per step",
                       "parallelism": f"replicas x{world}", "l2": "outputs of one step exceed the L2",
                       "autotune": tuned if tuned is not None else "off"},
            "per_mesh_loop": {"value": round(args.batch_meshes * world / (t_loop * 1e-3), 2), "unit": "meshes/s",
                              "ms_per_step": round(t_loop, 3)},
            "speedup_vs_loop": round(t_loop / t_batch, 3),
            "gvoxels_per_s": round(n_nodes * world / (t_batch * 1e-3) / 1e9, 3),
            "mtriangles_per_s": round(n_tris * world / (t_batch * 1e-3) / 1e6, 3),
            "identical_to_loop": bool(same), "gpu_launches": int(launches * steps), "clocks": clk.summary()}
    return line


SERVE_METRIC = "served voxelization (Poisson arrivals, 256-mesh mix shapes): sustained meshes/s and p50/p99 latency"


def _poisson(rate, n, rng):
    return np.cumsum(rng.exponential(1.0 / rate, size=n))


def _drive(submit, wait, pool, arrivals):
    """Submits pool[k % len(pool)] at arrivals[k] (seconds from start) from
    one thread and waits for the results in order from another; returns the
    latencies (s) and the span from the first arrival to the last result."""
    results = [None] * len(arrivals)
    lat = [0.0] * len(arrivals)
    done = [0.0]
    t0 = time.perf_counter() + 0.05

    def waiter():
        for k in range(len(arrivals)):
            while results[k] is None:
                time.sleep(0.0002)
            lat[k] = wait(results[k]) - (t0 + arrivals[k])
        done[0] = time.perf_counter()

    th = threading.Thread(target=waiter)
    th.start()
    for k, ta in enumerate(arrivals):
        dt = t0 + ta - time.perf_counter()
        if dt > 0:
            time.sleep(dt)
        results[k] = submit(pool[k % len(pool)])
    th.join()
    return lat, done[0] - t0


def run_served(args, world, rank, local):
    """Poisson request streams at several rates through the continuous-
    batching server, beside the plain path (one voxelization call per
    request, first come first served) under the same arrivals."""
    rates = [50, 200, 1000, 2000]
    rows = served_rows(args, local, rates, args.serve_seconds)
    top = rows[-1]
    line = {"metric": SERVE_METRIC, "value": top["served"]["meshes_per_s"], "unit": "meshes/s", "n_gpus": world,
            "steps": len(rates), "warmup": 1, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64+f32+u32", "data": "synthetic (seeded 256-mesh mix shapes, Poisson arrivals)",
            "config": {"workload": "LongNode with materials; admission by a 160 GB device-memory budget; 2 lanes",
                       "rates_req_s": rates, "seconds_per_rate": args.serve_seconds},
            "p50_ms": top["served"]["p50_ms"], "p99_ms": top["served"]["p99_ms"], "rates": rows}
    if rank == 0:
        print(json.dumps(line), flush=True)


def served_rows(args, local, rates, seconds):
    """Per rate: served and plain-path p50 / p99 latency and meshes/s."""
    import queue

    import torch

    from voxelizer_b200 import scenes
    from voxelizer_b200.api import LONG, Voxelizer
    from voxelizer_b200.serve import VoxelServer

    torch.cuda.set_device(local)
    # Default launch shapes: no tuning trials inside the timed request streams.
    from voxelizer_b200 import _lib
    _lib.set_autotune(0)
    pool = scenes.batch_mix(args.batch_meshes, seed=1)
    rng = np.random.default_rng(7)
    rows = []
    for rate in rates:
        n = int(min(args.serve_max_requests, max(50, rate * seconds)))
        arrivals = _poisson(rate, n, rng)
        # Served.
        with VoxelServer(budget_bytes=160 << 30, lanes=2, device=local) as srv:
            def submit(item):
                m, md = item
                return srv.submit(m.vertices, m.indices, m.materials, m.n_materials, size=md, node_type=LONG)

            def wait(req):
                req.wait()
                t = req.t_done
                srv.release(req)
                return t

            # Warm-up: the whole pool at once (the largest batches the lanes
            # can form), then the measured rate over the pool, so that the
            # lanes' batch buffers have grown before timing.
            _drive(submit, wait, pool, np.zeros(len(pool)))
            _drive(submit, wait, pool, _poisson(rate, min(len(pool), n), rng))
            lat_s, span_s = _drive(submit, wait, pool, arrivals)
            batches = srv.batches
        # Plain path: one worker, one call per request, in arrival order.
        q = queue.Queue()
        stream = torch.cuda.Stream()

        def worker():
            while True:
                item = q.get()
                if item is None:
                    return
                (m, md), box = item
                with Voxelizer(m.vertices, m.indices, m.materials, m.n_materials, node_type=LONG,
                               device=local) as v:
                    info = v.plan(1, md)
                    with torch.cuda.stream(stream):
                        out = torch.empty(int(info.bytes), dtype=torch.uint8, device="cuda")
                    v.voxelize_device(1, md, out, stream=stream.cuda_stream)
                box.append(time.perf_counter())

        th = threading.Thread(target=worker)
        th.start()

        def submit_plain(item):
            box = []
            q.put((item, box))
            return box

        def wait_plain(box):
            while not box:
                time.sleep(0.0002)
            return box[0]

        _drive(submit_plain, wait_plain, pool[:8], _poisson(1000, 16, rng))
        lat_p, span_p = _drive(submit_plain, wait_plain, pool, arrivals)
        q.put(None)
        th.join()
        pct = lambda a, p: round(float(np.percentile(np.asarray(a) * 1e3, p)), 3)  # noqa: E731
        rows.append({"rate_req_s": rate, "requests": n,
                     "served": {"meshes_per_s": round(n / span_s, 1), "p50_ms": pct(lat_s, 50),
                                "p99_ms": pct(lat_s, 99), "batches": batches},
                     "plain": {"meshes_per_s": round(n / span_p, 1), "p50_ms": pct(lat_p, 50),
                               "p99_ms": pct(lat_p, 99)}})
    return rows


def autotune(args, call, rounds=16):
    """With --autotune on: switch the launch-shape tuner on and make
    `rounds` untimed calls (3 candidate shapes x 3 samples, then 2
    material-key strategies x 3 samples settle a size bucket); returns the
    settled shapes (None when off)."""
    if args.autotune != "on":
        return None
    from voxelizer_b200 import _lib
    _lib.set_autotune(1)
    for _ in range(rounds):
        call()
    shapes = json.loads(_lib.autotune_state()[1])
    return shapes if len(shapes) <= 2 else {"buckets": len(shapes), "untimed_tuning_calls": rounds}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the short batched and served runs of the room line")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--workload", default="room", choices=["room", "batched", "served"],
                    help="room: the single-mesh headline; batched: the 256-mesh mix as one batch vs a per-mesh "
                         "loop; served: Poisson request streams through the continuous-batching server")
    ap.add_argument("--batch-meshes", type=int, default=256)
    ap.add_argument("--serve-seconds", type=float, default=1.5)
    ap.add_argument("--serve-max-requests", type=int, default=3000)
    ap.add_argument("--autotune", default="on", choices=["off", "on"],
                    help="on: tune launch shapes per size bucket in untimed calls before the warm-up "
                         "(results do not depend on the shapes)")
    ap.add_argument("--profile-run", type=int, default=0, metavar="MAXDIM",
                    help="no timing: voxelize the room scene at this maxDimension --steps times (a target for ncu)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    if args.profile_run:
        profile_run(args)
        return
    if args.workload == "batched":
        run_batched(args, world, rank, local)
        return
    if args.workload == "served":
        run_served(args, world, rank, local)
        return

    import torch

    from voxelizer_b200 import scenes
    from voxelizer_b200.api import LONG, Voxelizer

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    mesh = scenes.room_scene()
    vx = Voxelizer(mesh.vertices, mesh.indices, mesh.materials, mesh.n_materials, node_type=LONG, device=local)
    info = vx.plan(1, MAX_DIM)
    n_nodes = int(info.count)
    out = torch.empty(int(info.bytes), dtype=torch.uint8, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream
    tuned = autotune(args, lambda: (vx.voxelize_device(1, MAX_DIM, out, stream=sh), stream.synchronize()))
    for _ in range(args.warmup):
        vx.voxelize_device(1, MAX_DIM, out, stream=sh)
    stream.synchronize()
    launches = vx.last_launch_count()

    # Timed: profiling off (no stage events inside the timed calls).
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for i in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
            evs[i][0].record(stream)
            vx.voxelize_device(1, MAX_DIM, out, stream=sh)
            evs[i][1].record(stream)
        stream.synchronize()
    torch.cuda.synchronize()
    total_ms = sum(a.elapsed_time(b) for a, b in evs)
    if dist:
        total_ms = max_over_ranks(total_ms, dist)
        dist.barrier()
    ms = total_ms / args.steps
    value = replica_throughput(n_nodes, world, ms) / 1e9

    # Stage times from separate untimed passes with per-stage CUDA events: with
    # the stages one after another (each kernel's own time, for the roofline)
    # and as they run in the step (the timeline of the overlap).
    stage_acc = {}
    vx.set_profiling(True, serial=True)
    for _ in range(5):
        with torch.cuda.stream(stream):
            flush.zero_()
        vx.voxelize_device(1, MAX_DIM, out, stream=sh)
        for k, v in vx.stage_times().items():
            stage_acc.setdefault(k, []).append(v)
    vx.set_profiling(True)
    for _ in range(3):
        with torch.cuda.stream(stream):
            flush.zero_()
        vx.voxelize_device(1, MAX_DIM, out, stream=sh)
        timeline = vx.stage_timeline()
    vx.set_profiling(False)
    stream.synchronize()

    # e2e through the reference-facing entry with host buffers.
    pin_v = torch.from_numpy(mesh.vertices.reshape(-1)).pin_memory().numpy()
    pin_i = torch.from_numpy(mesh.indices.reshape(-1).view(np.int32)).pin_memory().numpy().view(np.uint32)
    pin_m = torch.from_numpy(mesh.materials).pin_memory().numpy()
    host_out = torch.empty(int(info.bytes), dtype=torch.uint8).pin_memory().numpy().view(np.uint16)
    e2e_ms = []
    for i in range(args.e2e_steps + 1):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        with Voxelizer(pin_v, pin_i, pin_m, mesh.n_materials, node_type=LONG, device=local) as v2:
            v2.voxelizeToNodesToRAM(MAX_DIM, out=host_out)
        torch.cuda.synchronize()
        if i > 0:
            e2e_ms.append(1e3 * (time.perf_counter() - t0))
    e2e = sorted(e2e_ms)[len(e2e_ms) // 2]   # median: the PCIe copy of a shared host varies
    if dist:
        e2e = max_over_ranks(e2e, dist)
    e2e_value = replica_throughput(n_nodes, world, e2e) / 1e9

    peak, peak_kind = peaks()
    stats = vx.last_stats()

    def median(name):
        v = sorted(stage_acc.get(name, [0.0]))
        return v[len(v) // 2]

    # Algorithmic bytes per launch of the two heaviest kernels.
    #  emit: the node grid written once, the pruned and surface bit grids read once.
    #  surface work: every partitioned triangle's record (64 B) and the edge
    #  functions its class tests (36 B for 2D boxes, 108 B for 3D boxes), and
    #  per hit an 8-byte hit-list entry and a 4-byte surface-word update
    #  (read and write).
    emit_bytes = n_nodes * 2 + 2 * n_nodes / 8
    st_tris = stats["surface_triangles"]
    surf_bytes = 64 * sum(st_tris) + 36 * st_tris[1] + 108 * st_tris[2] + 16 * stats["surface_hits"]
    kernels = [("emitNarrowKernel<LongNode>", emit_bytes, median("emit"), "emit_cartesian_long_room1024_bytes"),
               ("surfaceWorkKernel", surf_bytes, median("surface_work"), "surface_work_room1024_bytes")]
    roofs = []
    for name, nbytes, kms, tkey in kernels:
        ach = nbytes / (kms * 1e-3) / 1e9 if kms > 0 else None
        roofs.append({"bound": "hbm", "kernel": name, "achieved": round(ach, 1) if ach else None, "peak": peak,
                      "unit": "GB/s", "peak_kind": peak_kind, "frac": round(ach / peak, 4) if ach else None,
                      "traffic": ncu_traffic(tkey), "algorithmic_bytes": int(nbytes), "ms": round(kms, 4)})
    roofs.sort(key=lambda r: -r["ms"])   # the dominant kernel first
    path_bytes = 12 * mesh.n_vertices + 13 * mesh.n_triangles + n_nodes * 2
    line = {"metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64+f32+u32", "data": "synthetic (seeded room scene)",
            "config": dict(CONFIG), "parallelism": f"replicas x{world}",
            "autotune": tuned if tuned is not None else "off",
            "roofline": roofs[0],
            "roofline_next_kernel": roofs[1],
            "work": stats,
            "mtriangles_per_s": round(mesh.n_triangles * world / (ms * 1e-3) / 1e6, 1),
            "path_roofline": {"algorithmic_bytes": int(path_bytes),
                              "achieved": round(path_bytes / (ms * 1e-3) / 1e9, 1),
                              "frac": round(path_bytes / (ms * 1e-3) / 1e9 / peak, 4)},
            "stages_ms": {k: round(sorted(v)[len(v) // 2], 4) for k, v in stage_acc.items()},
            "stages_note": "stages_ms and the roofline ms: each stage alone (stages one after another); "
                           "stage_timeline_ms: the stages as they overlap in the timed step",
            "stage_timeline_ms": {k: [round(a, 3), round(b, 3)] for k, (a, b) in timeline.items() if a == a},
            "e2e": {"value": round(e2e_value, 3), "unit": UNIT, "ms_per_step": round(e2e, 3),
                    "h2d_bytes_per_step": int(12 * mesh.n_vertices + 13 * mesh.n_triangles),
                    "d2h_bytes_per_step": int(info.bytes)},
            "gpu_launches": int(launches * args.steps),
            "clocks": clk.summary()}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(mesh)
    if rank == 0 and world == 1 and not args.no_extras:
        # The batched and served forms of the target, in short runs: the
        # 256-mesh mix as one graph-replayed batch against the per-mesh loop,
        # and one Poisson rate through the server against the plain path.
        vx.close()
        del out, flush
        torch.cuda.empty_cache()
        bl = batched_line(args, 1, local, steps=10, warmup=3)
        line["batched"] = {k: bl[k] for k in ("value", "unit", "ms_per_step", "per_mesh_loop", "speedup_vs_loop",
                                               "identical_to_loop", "gvoxels_per_s", "mtriangles_per_s",
                                               "gpu_launches", "clocks")}
        line["batched"]["workload"] = bl["config"]["workload"]
        row = served_rows(args, local, [1000], 1.0)[0]
        line["served"] = {"rate_req_s": row["rate_req_s"], "requests": row["requests"], "unit": "meshes/s",
                          "served": row["served"], "plain": row["plain"],
                          "workload": "Poisson arrivals of the 256-mesh mix shapes, LongNode with materials, "
                                      "160 GB admission budget, 2 lanes"}
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
