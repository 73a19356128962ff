"""Parity of the CUDA path (through the C ABI) with the CPU oracle and with
the reference's own CUDA output (golden fixtures from tests/golden).

Rules (bit-exact; integer and bit work admits no tolerance):
  * bit arrays and boundary ids: identical;
  * materials: identical wherever the reference is deterministic.  Where
    triangles of different materials touch one node inside its winning
    triangle class the reference's plain stores race (src/voxelizer.cu:2988);
    there the oracle and the CUDA path pick the largest material and the
    golden comparison is skipped for those nodes (the oracle flags them).
"""

import hashlib
import json
import os

import numpy as np
import pytest

import cases as C
import oracle as O
from helpers import (CONFLICT_MAT, CONFLICT_RATIO, PARTIAL, RATIO_REF_TOL, RATIO_TOL, RATIO_UNSTABLE, bid_of,
                     bit_rows_mask, describe_diff, mat_of, masked, node_rows_mask, oracle_case, ratio_bad, ratio_of)
from voxelizer_b200.api import LONG, SHORT, Voxelizer
from voxelizer_b200.scenes import Mesh

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")
INDEX = json.load(open(os.path.join(GOLD, "index.json")))



@pytest.fixture(scope="module", autouse=True)
def _gpu():
    import torch
    assert torch.cuda.is_available(), "these tests need a CUDA device"


def make_voxelizer(c):
    m = C.mesh(c["mesh"])
    v = Voxelizer(m.vertices, m.indices, node_type=c["node_type"])
    if c["materials"]:
        v.setMaterials(m.materials, m.n_materials)
    return m, v


def run_gpu(c):
    m, v = make_voxelizer(c)
    with v:
        sp = c.get("space")
        if sp and sp[0] == "slice":
            out, info = v.voxelizeSliceToRAM(c["size"], sp[1], sp[2], c["vox"], c["mat"])
        elif sp:
            out, info = v.voxelizePartsToRAM(c["nodes"], c["size"], (sp[1], sp[2]), c["vox"], c["mat"])[sp[3]]
        elif c["nodes"]:
            out, info = v.voxelizeToNodesToRAM(c["size"], c["vox"], c["mat"])
        else:
            out, info = v.voxelizeToRAM(c["size"], c["vox"])
    return m, masked(c["node_type"], c["nodes"], out), info


FULL = sorted(n for n, e in INDEX.items() if "ref_error" not in e and C.BY_NAME[n]["store"] == "full")
DIGEST = sorted(n for n, e in INDEX.items() if "ref_error" not in e and C.BY_NAME[n]["store"] == "digest")


@pytest.mark.parametrize("name", FULL)
def test_small_cases(name):
    c = C.BY_NAME[name]
    m, got, info = run_gpu(c)
    assert info.dims == tuple(INDEX[name]["dims"])
    want, _, conf = oracle_case(c, m)
    want = masked(c["node_type"], c["nodes"], want)
    nt = c["node_type"]
    ratios = nt == PARTIAL and c["materials"]
    if ratios:
        # Same winning triangle per node; the ratio field within the oracle's
        # tolerance, everything else exact.
        low = np.uint64(0xFFFFFFFF)
        assert np.array_equal(got & low, want & low), "CUDA vs oracle: " + describe_diff(got & low, want & low)
        stable = np.nonzero((conf & RATIO_UNSTABLE) == 0)[0]
        bad = stable[ratio_bad(got[stable], want[stable], RATIO_TOL)]
        assert bad.size == 0, f"CUDA vs oracle: {bad.size} ratios differ: {ratio_of(got[bad[:5]])} vs " \
                              f"{ratio_of(want[bad[:5]])}"
    else:
        assert np.array_equal(got, want), "CUDA vs oracle: " + describe_diff(got, want, info.dims)
    gold = np.load(os.path.join(GOLD, name + ".npz"))["out"]
    if not c["nodes"]:
        keep = bit_rows_mask(name, info.dims)
        assert np.array_equal(got[keep], gold[keep]), "CUDA vs reference: " + describe_diff(got[keep], gold[keep])
        return
    rows, limit = node_rows_mask(name, info.dims)
    bg, bw = bid_of(nt, got), bid_of(nt, gold)
    assert np.array_equal(bg[rows], bw[rows]), "ids vs reference: " + describe_diff(bg[rows], bw[rows])
    assert np.count_nonzero(bg != bw) <= limit, "ids vs reference in the anomaly box"
    keep = (conf & CONFLICT_MAT) == 0
    gm, wm = mat_of(nt, got), mat_of(nt, gold)
    assert np.array_equal(gm[keep], wm[keep]), "materials vs reference: " + describe_diff(gm[keep], wm[keep])
    if ratios:
        # Against the reference's own ratio wherever a single triangle of the
        # winning class wrote the node (non-surface nodes hold exactly 0 or 1)
        # and no edge parameter sits at a branch point.
        sole = np.nonzero(((conf & (CONFLICT_RATIO | RATIO_UNSTABLE)) == 0) & rows)[0]
        bad = sole[ratio_bad(got[sole], gold[sole], RATIO_REF_TOL)]
        exact = int(np.count_nonzero((got >> np.uint64(32))[sole] == (gold >> np.uint64(32))[sole]))
        assert bad.size == 0, f"ratios vs reference: {bad.size} of {sole.size} beyond {RATIO_REF_TOL} " \
                              f"({exact} bit-identical): {ratio_of(got[bad[:5]])} vs {ratio_of(gold[bad[:5]])}"
    elif INDEX[name]["deterministic"]:
        assert np.array_equal(got[keep & rows], gold[keep & rows])


@pytest.mark.parametrize("name", DIGEST)
def test_full_size_digests(name):
    c = C.BY_NAME[name]
    _, got, info = run_gpu(c)
    e = INDEX[name]
    assert info.dims == tuple(e["dims"])
    if c["nodes"]:
        bid = bid_of(c["node_type"], got).astype(np.uint32)
        assert hashlib.sha256(bid.tobytes()).hexdigest() == e["bid_sha256"]
        assert int(np.count_nonzero(bid)) == e["n_solid"]
        if e["deterministic"]:
            assert hashlib.sha256(got.tobytes()).hexdigest() == e["sha256"]
    else:
        assert hashlib.sha256(got.tobytes()).hexdigest() == e["sha256"]


def test_repeat_calls_identical():
    c = C.BY_NAME["room_lite_long"]
    m, v = make_voxelizer(c)
    with v:
        a, _ = v.voxelizeToNodesToRAM(c["size"])
        b, _ = v.voxelizeToNodesToRAM(c["size"])
        bits, _ = v.voxelizeToRAM(c["size"])
    assert np.array_equal(a, b)
    assert bits.any()


def test_device_entry_matches_host_entry():
    import torch
    c = C.BY_NAME["torus_long"]
    m, v = make_voxelizer(c)
    with v:
        host, info = v.voxelizeToNodesToRAM(c["size"])
        dev = torch.empty(int(info.bytes), dtype=torch.uint8, device="cuda")
        s = torch.cuda.Stream()
        v.voxelize_device(1, c["size"], dev, stream=s.cuda_stream)
        s.synchronize()
        assert v.last_launch_count() > 0
    assert np.array_equal(dev.cpu().numpy().view(np.uint16), host)


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [0, 1])
def test_triangle_soup_pruning_matches_oracle(seed):
    """Random overlapping triangles (thin, self-intersecting solids whose
    pruning cascades over several passes) in many small yz subspaces: the
    node grid equals the oracle's bit for bit."""
    rng = np.random.default_rng(seed)
    n = 4000
    centres = rng.uniform(0.0, 1.0, size=(n, 1, 3))
    v = (centres + rng.normal(scale=0.04, size=(n, 3, 3))).reshape(-1, 3).astype(np.float32)
    f = np.arange(3 * n, dtype=np.uint32).reshape(n, 3)
    m = Mesh(v, f, None, 0)
    size, vox = 96, (1024, 8, 8)
    import torch

    for nt in (SHORT, LONG):
        with Voxelizer(m.vertices, m.indices, node_type=nt) as vx:
            got, info = vx.voxelizeToNodesToRAM(size, vox)
            pinned = torch.empty(int(info.bytes), dtype=torch.uint8).pin_memory().numpy().view(got.dtype)
            streamed, _ = vx.voxelizeToNodesToRAM(size, vox, out=pinned)
        want, oi, _ = O.voxelize(m, nt, 1, 0, size, vox)
        assert info.dims == tuple(oi.dims)
        assert np.array_equal(got, want), describe_diff(got, want, info.dims)
        assert np.array_equal(streamed, want)
        assert np.count_nonzero(bid_of(nt, got))


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["room_lite_long", "torus_short_splits", "ico4_partial_mat", "ico4_sfcc_mat"])
def test_pinned_host_output_matches(name):
    """A pinned host buffer takes the node array range by range while it is
    emitted (copies overlapped with the emission); the bytes equal the
    pageable path's."""
    import torch

    c = C.BY_NAME[name]
    m, v = make_voxelizer(c)
    with v:
        want, info = v.voxelizeToNodesToRAM(c["size"], c["vox"], c["mat"])
        pinned = torch.empty(int(info.bytes), dtype=torch.uint8).pin_memory().numpy().view(want.dtype)
        for _ in range(2):
            pinned[:] = 0
            got, _ = v.voxelizeToNodesToRAM(c["size"], c["vox"], c["mat"], out=pinned)
            assert got.ctypes.data == pinned.ctypes.data
            assert np.array_equal(masked(c["node_type"], 1, got), masked(c["node_type"], 1, want))
