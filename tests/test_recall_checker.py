"""The recall checkers against a plain brute force.

Recall@k of every form is scored by drpt_b200.recall.exact_knn_fp64 (GPU,
used by bench.py and the GPU tests) or oracle.exact_knn (CPU).  Both take
their candidates from an FP64 norm expansion; here they must return exactly
the neighbours of a brute force that computes every distance from
differences in FP64 and orders by (distance, index): on clustered float
rows, on small-integer rows where many distances tie exactly at the k-th
place, and on rows with exact duplicates (distance 0 to another point)."""
import numpy as np
import pytest

import oracle
from drpt_b200 import recall


def brute_force(X, queries, k):
    Xd = np.asarray(X, np.float64)
    idx = np.empty((len(queries), k), np.int64)
    dist = np.empty((len(queries), k), np.float64)
    ar = np.arange(len(Xd))
    for r, q in enumerate(queries):
        diff = Xd - Xd[q]
        d = np.sqrt(np.einsum("ij,ij->i", diff, diff))
        d[q] = np.inf
        o = np.lexsort((ar, d))[:k]
        idx[r], dist[r] = o, d[o]
    return idx, dist


def cases():
    rng = np.random.default_rng(11)
    centres = rng.uniform(0, 200, size=(20, 32))
    clustered = (centres[rng.integers(0, 20, 2000)] + rng.normal(0, 12, (2000, 32))).astype(np.float32)
    ties = rng.integers(0, 3, size=(1500, 6)).astype(np.float32)  # 3^6 cells: exact ties everywhere
    dup = rng.normal(0, 1, size=(1200, 16)).astype(np.float32)
    dup[600:900] = dup[:300]  # 300 exact duplicates
    return {"clustered": clustered, "integer_ties": ties, "duplicates": dup}


@pytest.mark.parametrize("name", ["clustered", "integer_ties", "duplicates"])
@pytest.mark.parametrize("k", [10, 20])
def test_cpu_checkers_equal_brute_force(name, k):
    X = cases()[name]
    q = recall.sample_queries(len(X), 300, seed=3)
    want_i, want_d = brute_force(X, q, k)
    got_i, got_d = oracle.exact_knn(X, q, k)
    assert np.array_equal(got_i, want_i), name
    np.testing.assert_allclose(got_d, want_d, rtol=1e-12, atol=0)
    # the GPU checker's logic, run by torch on the CPU
    got_i, got_d = recall.exact_knn_fp64(X, q, k, device="cpu")
    assert np.array_equal(got_i, want_i), name
    np.testing.assert_allclose(got_d, want_d, rtol=1e-12, atol=0)


def test_integer_ties_reach_the_fallback():
    # the tie case must really exercise the all-points path: rows with more
    # than k + 16 points at or below the k-th distance, where candidates
    # from the norm expansion alone could miss the lowest tied indices
    X = cases()["integer_ties"]
    q = recall.sample_queries(len(X), 300, seed=3)
    _, d = brute_force(X, q, 10)
    Xd = X.astype(np.float64)
    crowded = 0
    for r, p in enumerate(q):
        dd = np.sqrt(((Xd - Xd[p]) ** 2).sum(1))
        dd[p] = np.inf
        crowded += int((dd <= d[r, -1]).sum() > 10 + 16)
    assert crowded >= 20


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["clustered", "integer_ties", "duplicates"])
def test_gpu_checker_equals_brute_force(name):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    X = cases()[name]
    q = recall.sample_queries(len(X), 300, seed=3)
    want_i, want_d = brute_force(X, q, 10)
    got_i, got_d = recall.exact_knn_fp64(torch.from_numpy(X).cuda(), q, 10)
    assert np.array_equal(got_i, want_i), name
    np.testing.assert_allclose(got_d, want_d, rtol=1e-12, atol=0)
