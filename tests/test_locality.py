"""The locality relabelling (drpt_locality_slots, host code in the library)
against the reference's own -locality 1 runs in the golden fixtures: the
leaves of every tree must land in the same slots.  No GPU needed."""
import ctypes
import glob
import os

import numpy as np
import pytest

from drpt_b200 import _lib
from tests.conftest import GOLDEN

CASES = [c for c in sorted(glob.glob(os.path.join(GOLDEN, "case_*.npz")))
         if "locality_final_order" in np.load(c).files]


def _global_leaves(order, offsets, nleaf):
    """Every tree's global leaves from its final leaves (each global leaf
    holds n_final / nleaf consecutive final leaves), members ascending."""
    T, n = order.shape
    per = (offsets.shape[1] - 1) // nleaf
    g_order = np.empty((T, n), np.int32)
    g_off = np.zeros((T, nleaf + 1), np.int32)
    for t in range(T):
        w = 0
        for j in range(nleaf):
            m = np.sort(order[t, offsets[t, j * per]:offsets[t, (j + 1) * per]])
            g_order[t, w:w + len(m)] = m
            w += len(m)
            g_off[t, j + 1] = w
    return g_order, g_off


def _slots(order, offsets, nleaf):
    L = _lib.load()
    T, n = order.shape
    slots = np.full((nleaf, T), -1, np.int32)
    so, sf = np.empty_like(order), np.empty_like(offsets)
    st = L.drpt_locality_slots(order.ctypes.data, offsets.ctypes.data, n, T, nleaf,
                               slots.ctypes.data, so.ctypes.data, sf.ctypes.data)
    return st, slots, so, sf


@pytest.mark.parametrize("case", CASES, ids=lambda c: os.path.basename(c)[5:-4])
def test_slots_match_reference(case):
    g = np.load(case)
    T, gd = int(g["ntrees"]), int(g["gd"])
    nleaf = 1 << (gd - 1)
    go, gf = _global_leaves(g["final_order"], g["final_offsets"], nleaf)
    lo, lf = _global_leaves(g["locality_final_order"], g["locality_final_offsets"], nleaf)
    st, slots, so, sf = _slots(go, gf, nleaf)
    _lib.check(st)
    for t in range(T):
        key = {tuple(go[t, gf[t, j]:gf[t, j + 1]]): j for j in range(nleaf)}
        want = [key[tuple(lo[t, lf[t, k]:lf[t, k + 1]])] for k in range(nleaf)]
        assert slots[:, t].tolist() == want
        assert sorted(want) == list(range(nleaf))
    # the rearranged leaves are the reference's slot-ordered global leaves
    assert np.array_equal(sf, lf) and np.array_equal(so, lo)


def test_locality_argument_checks():
    g = np.load(CASES[0])
    gd = int(g["gd"])
    nleaf = 1 << (gd - 1)
    go, gf = _global_leaves(g["final_order"], g["final_offsets"], nleaf)
    bad = gf.copy()
    bad[0, -1] -= 1  # offsets no longer cover the points
    assert _slots(go, bad, nleaf)[0] == 1
    bad = go.copy()
    bad[0, 0] = go.shape[1]  # a point id out of range
    assert _slots(bad, gf, nleaf)[0] == 1
    assert _slots(go, gf, nleaf + 1)[0] == 1  # not a power of two
