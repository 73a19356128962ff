"""Shared helpers for the parity tests: node field extraction, the
comparison rule for materials (nodes whose winning surface class saw more
than one material are compared only by boundary id) and for the PartialNode
ratio (a float field: NaN positions equal, values within a tolerance where
the oracle's plain IEEE arithmetic is compared with the reference's
contracted FP32)."""

from __future__ import annotations

import numpy as np

SHORT, LONG, PARTIAL, SHORT_FCC, LONG_FCC = range(5)


def padding_mask(node_type, nodes):
    if not nodes:
        return None
    if node_type == LONG_FCC:
        return np.uint32(0x00FFFFFF)
    if node_type == PARTIAL:
        return np.uint64(0xFFFFFFFF0000FFFF)
    return None


def bid_of(node_type, a):
    return {SHORT: lambda x: x & 31, LONG: lambda x: x & 0xFF, PARTIAL: lambda x: x & 0xFF,
            SHORT_FCC: lambda x: x & 4095, LONG_FCC: lambda x: x & 0xFFFF}[node_type](a)


def mat_of(node_type, a):
    return {SHORT: lambda x: x >> 5, LONG: lambda x: x >> 8, PARTIAL: lambda x: (x >> 8) & 0xFF,
            SHORT_FCC: lambda x: x >> 12, LONG_FCC: lambda x: (x >> 16) & 0xFF}[node_type](a)


def masked(node_type, nodes, a):
    pm = padding_mask(node_type, nodes)
    return a & pm if pm is not None else a


def describe_diff(a, b, dims=None, limit=5):
    d = np.nonzero(a != b)[0]
    msg = f"{d.size} of {a.size} elements differ"
    if d.size and dims is not None:
        X, Y, _ = dims
        pts = [(int(i % X), int(i // X % Y), int(i // (X * Y)), int(a[i]), int(b[i])) for i in d[:limit]]
        msg += f"; first (x, y, z, got, want): {pts}"
    return msg


# Conflict bits of the oracle (orc_voxelize's conflict_out).
CONFLICT_MAT, CONFLICT_RATIO, RATIO_UNSTABLE = 1, 2, 4

# |ratio(oracle) - ratio(reference or CUDA)|: the oracle evaluates the
# reference's FP32 operation order without multiply-add contraction and with
# 1 / sqrtf in place of rsqrtf.
RATIO_TOL = 2e-3

# |ratio(CUDA) - ratio(reference)| where one triangle decides the node.  Both
# evaluate the same FP32 operation order with nvcc's contraction, but the
# reference's contraction depends on the kernel its inline function lands in
# (the reference's own function compiled into another kernel reproduces its
# in-kernel results on 91% of such nodes), so the last bits are not pinned.
# Most nodes agree bit for bit; the volume sums pyramids over rotated
# absolute coordinates, and a few configurations amplify last-bit
# differences to a few 1e-4 (seen on 2 of 35,151 torus surface nodes).
RATIO_REF_TOL = 1e-3


def ratio_of(a):
    """PartialNode ratio field (bytes 4-7) as float32."""
    return (np.asarray(a, dtype=np.uint64) >> np.uint64(32)).astype(np.uint32).view(np.float32)


def ratio_bad(got, want, tol):
    """Indices where the ratios differ: NaN in one only, or |diff| > tol."""
    g, w = ratio_of(got), ratio_of(want)
    gn, wn = np.isnan(g), np.isnan(w)
    with np.errstate(invalid="ignore"):
        far = np.abs(g.astype(np.float64) - w.astype(np.float64)) > tol
    return np.nonzero((gn != wn) | (~gn & ~wn & far))[0]


def oracle_case(c, m, want_conflicts=True):
    """The oracle's output for a golden case, device spaces included: the
    partition of a slice or devConfig case comes from the planned grid; a
    slice past the grid is the zero array (sliceOOB)."""
    import cases as C
    import oracle as O
    part, oob, rot = None, False, C.turned(c)
    if c.get("space"):
        pl = O.plan(m, c["node_type"], c["nodes"], c["size"], c["vox"], rotate_x=rot)
        ry, rz = int(pl.resolution[1]), int(pl.resolution[2])
        part, oob = C.partition(c, ry, rz), C.slice_oob(c, ry, rz)
    out, info, conf = O.voxelize(m, c["node_type"], c["nodes"], c["materials"], c["size"], c["vox"], c["mat"],
                                 want_conflicts=want_conflicts, part=part, rotate_x=rot)
    if oob:
        out[:] = 0
        if conf is not None:
            conf[:] = 0
    return out, info, conf


# Rows of golden bit arrays where the reference's own output lost its
# crossings, keyed by case: (y, z) allocation rows.  generateVoxelization
# (src/voxelizer.cu:1321-1333) initialises its shared loop flags and segment
# arrays and then tests the loop condition without a __syncthreads(), so a
# thread can read another warp's stale flag and skip every triangle of its
# tile; its voxel row then gets no crossings at all.  The row's neighbours,
# the same voxel in the full-grid golden and this project's output all have
# the crossings.
REF_ANOMALY_ROWS = {"room_lite_bits_part13_1": [(76, 24)]}

# Node-grid counterpart: a box of node rows (y range, z range, inclusive) of
# a golden node grid where the reference's solid bits differ from the
# restated algorithm's, and the most boundary ids that differ inside it.
# Materials and surface nodes are identical in both boxes.
#  * stress_partial_mat (8,120 triangles, 96x80x80 PartialNodes): the
#    reference's rows y 74-75 x z 59-60 (one 4x4 solid tile) hold solid runs
#    at x 14-15, 18-19, 43-44, 46-47 and 54 that no triangle crossing those
#    rows produces; pruning spreads them to 45 boundary ids.
#  * stress_full_sfcc (20,120 triangles, 192x68x136 ShortFCCNodes): three
#    node rows of sub-lattice 1 are solid from x 132 to the row's end in the
#    reference only; 679 boundary ids differ around them.
# Both sit where a generation edge function of a 45-degree edge is exactly
# 0 at a voxel centre (triangles 8091 and 18257), but the same tie in
# stress_sfcc_mat (triangle 7364) resolves the other way in the reference,
# so no contraction mode of the FP64 solid path reproduces all three; the
# reference's two runs agree on the boundary ids of every case.
REF_ANOMALY_NODE_BOX = {"stress_partial_mat": ((73, 76), (58, 60), 45),
                        "stress_full_sfcc": ((49, 52), (99, 104), 679)}


def node_rows_mask(name, dims):
    """Boolean mask over the nodes of a golden node grid: False inside the
    case's anomaly box (REF_ANOMALY_NODE_BOX), and that box's bound on the
    number of boundary ids that may differ inside it (0 without a box)."""
    X, Y, Z = dims
    keep = np.ones(X * Y * Z, dtype=bool)
    box = REF_ANOMALY_NODE_BOX.get(name)
    if box is None:
        return keep, 0
    (y0, y1), (z0, z1), limit = box
    k = keep.reshape(Z, Y, X)
    k[z0:z1 + 1, y0:y1 + 1, :] = False
    return keep, limit


def bit_rows_mask(name, dims):
    """Boolean mask over the words of a bit array: False on anomaly rows."""
    X, Y, Z = dims
    ipx = X // 32
    keep = np.ones(ipx * Y * Z, dtype=bool)
    for y, z in REF_ANOMALY_ROWS.get(name, []):
        r = (z * Y + y) * ipx
        keep[r:r + ipx] = False
    return keep
