"""Shared helpers for the parity tests: node field extraction and the
comparison rule for materials (material resolution)."""

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
