"""The CPU oracle against the reference's own CUDA output (golden fixtures
produced by tests/golden/make_golden.py from oracle/_ref on a B200), plus
properties of the restated algorithm.  CPU only."""

import json
import os

import numpy as np
import pytest

import cases as C
import oracle as O
from helpers import (CONFLICT_MAT, CONFLICT_RATIO, PARTIAL, RATIO_TOL, RATIO_UNSTABLE, bid_of, describe_diff,
                     bit_rows_mask, mat_of, masked, node_rows_mask, oracle_case, ratio_bad, ratio_of)

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")
INDEX = json.load(open(os.path.join(GOLD, "index.json")))
FULL = sorted(n for n, e in INDEX.items() if "ref_error" not in e and C.BY_NAME[n]["store"] == "full")


@pytest.mark.parametrize("name", FULL)
def test_oracle_matches_reference(name):
    c = C.BY_NAME[name]
    m = C.mesh(c["mesh"])
    out, info, conf = oracle_case(c, m)
    out = masked(c["node_type"], c["nodes"], out)
    gold = np.load(os.path.join(GOLD, name + ".npz"))["out"]
    if not c["nodes"]:
        keep = bit_rows_mask(name, tuple(info.dims))
        assert np.array_equal(out[keep], gold[keep]), describe_diff(out[keep], gold[keep])
        return
    nt = c["node_type"]
    rows, limit = node_rows_mask(name, tuple(info.dims))
    bo, bg = bid_of(nt, out), bid_of(nt, gold)
    assert np.array_equal(bo[rows], bg[rows]), describe_diff(bo[rows], bg[rows])
    assert np.count_nonzero(bo != bg) <= limit
    keep = (conf & CONFLICT_MAT) == 0
    assert np.array_equal(mat_of(nt, out)[keep], mat_of(nt, gold)[keep])
    if nt == PARTIAL and c["materials"]:
        # The ratio field: within the restatement's tolerance wherever one
        # triangle of the winning class decides it.
        sole = np.nonzero(((conf & (CONFLICT_RATIO | RATIO_UNSTABLE)) == 0) & rows)[0]
        bad = sole[ratio_bad(out[sole], gold[sole], RATIO_TOL)]
        assert bad.size == 0, f"{bad.size} ratios differ, e.g. {ratio_of(out[bad[:5]])} vs {ratio_of(gold[bad[:5]])}"
        low = np.uint64(0xFFFFFFFF)
        assert np.array_equal((out & low)[keep & rows], (gold & low)[keep & rows])
    elif INDEX[name]["deterministic"]:
        assert np.array_equal(out[keep & rows], gold[keep & rows])
    if not INDEX[name]["deterministic"]:
        # Every node the reference wrote differently on its two runs must be
        # a node the oracle flags as contested.
        g2 = np.load(os.path.join(GOLD, name + ".npz"))["out2"]
        diff = np.nonzero(gold != g2)[0]
        assert np.all(conf[diff] != 0)


def test_fcc_neighbourhood_is_symmetric():
    """calculateFCCBoundaries updates nodes in place (src/voxelizer.cu:1929-2048);
    the result is order independent only if neighbour k of A has A as its
    neighbour.  Checked over a small grid by brute force."""
    NX, NY, NZ = 8, 5, 6
    offs = []

    def nbrs(x, y, z):
        out = []
        left, right, inn, outy = x > 0, x < NX - 1, y > 0, y < NY - 1
        down, up, xe = z > 0, z < NZ - 1, (x + z) % 2 == 0
        cin, cout = (xe and inn) or not xe, (not xe and outy) or xe
        ym, yp = (y - 1 if xe else y), (y if xe else y + 1)
        if down and cin: out.append((x, ym, z - 1))
        if down and left: out.append((x - 1, y, z - 1))
        if down and right: out.append((x + 1, y, z - 1))
        if down and cout: out.append((x, yp, z - 1))
        if left and cin: out.append((x - 1, ym, z))
        if right and cin: out.append((x + 1, ym, z))
        if left and cout: out.append((x - 1, yp, z))
        if right and cout: out.append((x + 1, yp, z))
        if up and cin: out.append((x, ym, z + 1))
        if up and left: out.append((x - 1, y, z + 1))
        if up and right: out.append((x + 1, y, z + 1))
        if up and cout: out.append((x, yp, z + 1))
        return out

    for x in range(NX):
        for y in range(NY):
            for z in range(NZ):
                for q in nbrs(x, y, z):
                    assert (x, y, z) in nbrs(*q)
                    offs.append(q)
    assert offs


def test_pruning_is_split_ordered():
    """With small yz splits the pruned set differs from a single split only
    near split boundaries, and both equal the reference (golden)."""
    c = C.BY_NAME["ico3_long_splits"]
    m = C.mesh(c["mesh"])
    a, _, _ = O.voxelize(m, c["node_type"], 1, 0, c["size"], c["vox"], c["mat"])
    b, info, _ = O.voxelize(m, c["node_type"], 1, 0, c["size"], (c["vox"][0], 512, 512), c["mat"])
    assert a.shape == b.shape and (bid_of(1, a) > 0).sum() > 0
    X, Y, Z = info.dims
    diff = np.nonzero(a != b)[0]
    ys, zs = diff // X % Y, diff // (X * Y)
    ends = [16 * k for k in range(Y // 16 + 2)]
    # Every difference sits on or next to a 16-row split boundary.
    near = lambda v: min(abs(int(v) - e) for e in range(0, max(Y, Z) + 16, 1) if e % 16 in (0,)) <= 2
    assert all(near(y) or near(z) for y, z in zip(ys, zs))
