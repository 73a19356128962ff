"""The exclusive scan that sizes every work list (vxb_scan_counts): offsets
equal to a host prefix sum, and the 2^32 overflow flag for sums that wrap
inside one thread's items, inside one 4096-count tile, and across tiles."""

import ctypes

import numpy as np
import pytest

from voxelizer_b200 import _lib


def _scan(counts):
    import torch

    c = torch.from_numpy(np.asarray(counts, np.uint32).view(np.int32)).cuda()
    off = torch.zeros(len(counts) + 1, dtype=torch.int32, device="cuda")
    total, overflow = ctypes.c_uint32(), ctypes.c_uint32()
    _lib.check(_lib.lib().vxb_scan_counts(ctypes.c_void_p(c.data_ptr()), len(counts), ctypes.c_void_p(off.data_ptr()),
                                          ctypes.byref(total), ctypes.byref(overflow), None))
    return off.cpu().numpy().view(np.uint32), total.value, overflow.value


@pytest.mark.gpu
@pytest.mark.parametrize("n", [0, 1, 4095, 4096, 4097, 10_000, 3 * 4096 * 1024 + 17])
def test_offsets_match_host_prefix_sum(n):
    rng = np.random.default_rng(n)
    counts = rng.integers(0, 300, n, dtype=np.uint32)
    off, total, overflow = _scan(counts)
    want = np.zeros(n + 1, np.uint64)
    want[1:] = np.cumsum(counts, dtype=np.uint64)
    assert overflow == 0
    assert total == int(want[-1])
    assert np.array_equal(off.astype(np.uint64), want)


@pytest.mark.gpu
@pytest.mark.parametrize("name,counts,flag", [
    # one thread's four items sum to 2^32
    ("thread", [1 << 31, 1 << 31, 0, 0], 1),
    # one 4096-count tile sums to 2^32 + 4096
    ("tile", [(1 << 20) + 1] * 4096, 1),
    # two tiles of 2^31 each: the carry reaches 2^32
    ("tiles", [1 << 19] * 8192, 1),
    # exactly 2^32 - 1: the flag is set from there on
    ("edge", [0xFFFFFFFF], 1),
    # 2^32 - 8192 over two tiles: no overflow
    ("below", [524287] * 8192, 0),
])
def test_overflow_flag(name, counts, flag):
    off, total, overflow = _scan(counts)
    assert overflow == flag, name
    if not flag:
        want = np.zeros(len(counts) + 1, np.uint64)
        want[1:] = np.cumsum(np.asarray(counts, np.uint64))
        assert total == int(want[-1])
        assert np.array_equal(off.astype(np.uint64), want)
