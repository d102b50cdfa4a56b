"""Comparison of k-NN lists "up to exact-distance ties".

The reference orders each leaf row with std::sort on distance only
(mdrpt.cpp:162-166) and merges trees with std::merge + an adjacent
std::unique by index (mdrpt.cpp:186-197).  Equal distances therefore come out
in an order the standard leaves unspecified, and a tie can even leave the
same neighbour twice in a list.  The library orders by (distance, index) and
removes every duplicate.  Two lists agree when:

* the distance sequences of their first k entries are identical, bit for
  bit, and
* every entry closer than the smallest tied distance has the same index.

Entries at or beyond the first tied distance may differ in index (and, when
a tie straddles a per-tree cut of 2k, in which equal-distance candidate was
kept); such points are counted as tie-affected.
"""
from __future__ import annotations

import numpy as np


def reference_first_k(ref_idx: np.ndarray, ref_dist: np.ndarray, k: int):
    """Each point's first k entries (k may exceed the nn of the run, to look
    past the cut) of the reference's merged list after dropping the point
    itself and repeated indices (first occurrence kept)."""
    n = ref_idx.shape[0]
    out_i = np.full((n, k), -1, np.int64)
    out_d = np.full((n, k), np.inf, np.float32)
    for p in range(n):
        ri, rd = ref_idx[p], ref_dist[p]
        m = (ri != p) & (ri >= 0)
        ri, rd = ri[m], rd[m]
        _, first = np.unique(ri, return_index=True)
        keep = np.sort(first)[:k]
        out_i[p, :len(keep)] = ri[keep]
        out_d[p, :len(keep)] = rd[keep]
    return out_i, out_d


def _first_tie(d: np.ndarray) -> float:
    """Smallest finite distance value that occurs more than once in d."""
    d = d[np.isfinite(d)]
    if len(d) < 2:
        return np.inf
    s = np.sort(d)
    eq = s[1:] == s[:-1]
    return float(s[1:][eq].min()) if eq.any() else np.inf


def compare(ref_i: np.ndarray, ref_d: np.ndarray, idx: np.ndarray, dist: np.ndarray,
            ref_tail_d: np.ndarray | None = None) -> dict:
    """ref_i/ref_d and idx/dist: (n, k).  ref_tail_d (n, w>=k), optional, the
    reference distances beyond k used to detect a tie across the k cut.
    Returns counts of exact, tie-affected and failing points."""
    n, k = idx.shape
    exact = tie = 0
    fails = []
    for p in range(n):
        if np.array_equal(ref_i[p], idx[p]) and np.array_equal(ref_d[p], dist[p]):
            exact += 1
            continue
        if not np.array_equal(ref_d[p], dist[p]):
            v = min(_first_tie(ref_d[p]), _first_tie(dist[p]))
            if ref_tail_d is not None:
                v = min(v, _first_tie(ref_tail_d[p]))
            # distances may diverge only at or beyond a tie
            lo = (ref_d[p] < v) | (dist[p] < v)
            if np.isfinite(v) and np.array_equal(ref_d[p][lo], dist[p][lo]) and \
                    np.array_equal(ref_i[p][lo], idx[p][lo]):
                tie += 1
            else:
                fails.append(p)
            continue
        v = min(_first_tie(ref_d[p]), _first_tie(dist[p]))
        if ref_tail_d is not None:
            v = min(v, _first_tie(ref_tail_d[p]))
        lo = ref_d[p] < v
        if np.array_equal(ref_i[p][lo], idx[p][lo]):
            tie += 1
        else:
            fails.append(p)
    return {"exact": exact, "tie": tie, "fail": len(fails), "fail_points": fails[:10]}
