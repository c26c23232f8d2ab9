"""The bank-aware link order of the time step's link streams (bank_deal.cu), on the host.

Each node keeps its links, only their slots change: the small links stay in the slots
[0, ij_count_small) and the other links in [ij_count_small, ij_count), every link exactly once,
padding after.  Within a slot, the lanes that read the tile halo together (16 for 8-byte loads,
8 for 16-byte loads) take links in distinct bank groups (local position mod the group size)
wherever a matching allows it.
"""
import ctypes as C
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "..", "sunset_viscoelastic_b200", "lib", "libsunset_hostcheck.so")


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB):
        from sunset_viscoelastic_b200 import build
        build.build()
    L = C.CDLL(LIB)
    ip = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
    up = np.ctypeslib.ndpointer(np.uint16, flags="C_CONTIGUOUS")
    L.sunset_hostcheck_deal.argtypes = [C.c_int, up, ip, ip, ip, ip, C.c_int, ip]
    return L


def deal(L, group, pos, small, large):
    soff = np.zeros(33, np.int32)
    loff = np.zeros(33, np.int32)
    soff[1:] = np.cumsum([len(s) for s in small])
    loff[1:] = np.cumsum([len(s) for s in large])
    width = max(len(a) + len(b) for a, b in zip(small, large))
    width = (width + 1) & ~1
    chosen = np.full(max(width, 1) * 32, -7, np.int32)
    flat = lambda ls: np.array([e for s in ls for e in s] or [0], np.int32)
    L.sunset_hostcheck_deal(group, pos, flat(small), soff, flat(large), loff, width, chosen)
    return chosen[: width * 32].reshape(width, 32)


@pytest.mark.parametrize("group", [8, 16])
@pytest.mark.parametrize("seed", range(6))
def test_every_link_once_in_its_range(lib, group, seed):
    rng = np.random.default_rng(seed)
    W = int(rng.integers(1, 90))
    e = 0
    small, large = [], []
    for lane in range(32):
        c = int(rng.integers(0, W + 1)) if lane < 28 or seed % 2 else 0
        cs = int(rng.integers(0, c + 1))
        ids = rng.permutation(np.arange(e, e + c)).tolist()
        e += c
        small.append(ids[:cs])
        large.append(ids[cs:])
    pos = rng.integers(0, 3000, size=max(e, 1)).astype(np.uint16)
    pos[rng.random(pos.size) < 0.1] |= np.uint16(2 << 14)  # mirror codes ride in the top bits
    ch = deal(lib, group, pos, small, large)
    for lane in range(32):
        cs, c = len(small[lane]), len(small[lane]) + len(large[lane])
        col = ch[:, lane]
        assert sorted(col[:cs].tolist()) == sorted(small[lane])
        assert sorted(col[cs:c].tolist()) == sorted(large[lane])
        assert np.all(col[c:] == -1)


@pytest.mark.parametrize("group", [8, 16])
def test_distinct_banks_where_every_lane_can_take_any(lib, group):
    """Every lane holds one link in each bank group: the first slot of every group of lanes
    takes `group` distinct bank groups, where the reference order would repeat one."""
    rng = np.random.default_rng(11)
    small, pos, e = [], [], 0
    for lane in range(32):
        banks = np.arange(group)
        # the reference order puts bank 3 first on every lane
        order = [3] + [b for b in rng.permutation(banks).tolist() if b != 3]
        ids = list(range(e, e + group))
        e += group
        small.append(ids)
        for b in order:
            pos.append(int(rng.integers(0, 200)) * group + b)
    pos = np.array(pos, np.uint16)
    ch = deal(lib, group, pos, small, [[] for _ in range(32)])
    for h in range(32 // group):
        lanes = range(group * h, group * (h + 1))
        first = [int(pos[ch[0, r]]) % group for r in lanes]
        assert len(set(first)) == group, first
