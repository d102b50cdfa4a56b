"""Parity with the reference at the workloads' own sizes (fixtures made by
tests/golden/make_scale_golden.py from the reference binary, one rank and one
thread):

* the ubyte workload at full size, 60,000 x 784 uint8, 8 trees, nn = 10,
  -locality 1: every tree's final leaves (in the locality pass's slot order)
  bit for bit, and the edge list (nn - 1 neighbours per point) equal up to
  exact-distance ties;
* the fbin workload's distribution at 131,072 x 128 float32, 16 trees,
  nn = 10: final leaves bit for bit, edge list equal per point (by hash);
* the ubyte workload with the generator's default spread, where the
  reference stops with std::length_error: the library returns an error
  status instead.

The CPU tests pin the oracle (the C++ restatement) to the same fixtures; the
GPU tests run the CUDA path through the C ABI."""
from __future__ import annotations

import hashlib
import os

import numpy as np
import pytest

import oracle
from drpt_b200 import MDRPT, DrptError, build_graph, global_depth, synth
from tests import knn_compare
from tests.conftest import GOLDEN

HASH_MUL = np.uint64(0x9E3779B97F4A7C15)


def _fixture(name: str):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


def _rows(g) -> np.ndarray:
    params = eval(str(g["gen_params"]), {"__builtins__": {}})  # a literal dict
    X = getattr(synth, str(g["gen"]))(int(g["n"]), int(g["d"]), **params)
    sha = hashlib.sha256(np.ascontiguousarray(X).tobytes()).hexdigest()
    assert sha == str(g["rows_sha256"]), "the seeded generator no longer gives the fixture's rows"
    return X


def _leaf_shas(order: np.ndarray, offsets: np.ndarray) -> list[str]:
    out = []
    for t in range(order.shape[0]):
        h = hashlib.sha256(np.ascontiguousarray(order[t], np.int32).tobytes())
        h.update(np.ascontiguousarray(offsets[t], np.int32).tobytes())
        out.append(h.hexdigest())
    return out


def _edge_hash(ids: np.ndarray) -> np.ndarray:
    ids = np.asarray(ids, np.int64)
    h = np.zeros(ids.shape[0], np.uint64)
    mul = np.uint64(1)
    with np.errstate(over="ignore"):
        for j in range(ids.shape[1]):
            mul = mul * HASH_MUL
            h = h + (ids[:, j] + 1).astype(np.uint64) * mul
    return h


def _check_edges_up_to_ties(X, ref_ids: np.ndarray, idx: np.ndarray, dist: np.ndarray) -> dict:
    """ref_ids: (n, nn-1) reference edge list; idx/dist: (n, nn) ours.  Points
    whose first nn-1 ids differ must differ only at or beyond an exact
    distance tie; the reference's distances of those points are recomputed
    with the oracle's distance (the reference's arithmetic)."""
    k = ref_ids.shape[1]
    bad = np.nonzero((ref_ids.astype(np.int64) != idx[:, :k]).any(axis=1))[0]
    if len(bad) == 0:
        return {"exact": len(idx), "tie": 0, "fail": 0}
    rd = np.array([[oracle.distance(X[q], X[p]) if q >= 0 else np.inf for q in ref_ids[p]]
                   for p in bad], np.float32)
    res = knn_compare.compare(ref_ids[bad].astype(np.int64), rd, idx[bad, :k].astype(np.int64),
                              dist[bad, :k], dist[bad])
    res["exact"] += len(idx) - len(bad)
    return res


def _check_edge_hash(g, idx: np.ndarray, dist: np.ndarray) -> dict:
    nn = int(g["nn"])
    bad = np.nonzero(_edge_hash(idx[:, :nn - 1]) != g["edge_hash"])[0]
    # a differing point must have an exact tie among its first nn distances
    tie = [p for p in bad if (np.diff(dist[p, :nn]) == 0).any()]
    sp = g["sample_points"]
    assert np.array_equal(idx[sp, :nn - 1], g["sample_edge_ids"]) or len(bad) > 0
    return {"differ": len(bad), "tie": len(tie), "fail": len(bad) - len(tie)}


# ---------------------------------------------------------------- oracle (CPU)
@pytest.mark.slow
def test_oracle_fbin_131k_equals_reference():
    g = _fixture("scale_c2_f32")
    X = _rows(g)
    seeds = g["seeds"]
    o = oracle.build(X, int(g["ntrees"]), int(g["nn"]), int(seeds[0]), local_seeds=seeds[1:])
    assert o["status"] == 0
    assert o["info"].global_depth == int(g["gd"]) and o["info"].local_depth == int(g["ld"])
    assert _leaf_shas(o["final_order"], o["final_offsets"]) == list(g["leaf_sha256"])
    res = _check_edge_hash(g, o["knn_idx"], o["knn_dist"])
    assert res["fail"] == 0, res


@pytest.mark.slow
def test_oracle_ubyte_60k_equals_reference():
    g = _fixture("scale_c1_u8")
    X = _rows(g)
    seeds = g["seeds"]
    o = oracle.build(X, int(g["ntrees"]), int(g["nn"]), int(seeds[0]), local_seeds=seeds[1:])
    assert o["status"] == 0
    res = _check_edges_up_to_ties(X, g["edge_ids"], o["knn_idx"], o["knn_dist"])
    assert res["fail"] == 0, res
    assert res["tie"] <= 0.01 * X.shape[0], res


# ---------------------------------------------------------------- CUDA path
@pytest.fixture(scope="module")
def torch():
    import torch as _t
    if not _t.cuda.is_available():
        pytest.skip("no CUDA device")
    return _t


def _mdrpt(g, X, locality: bool):
    n, d = X.shape
    td, _ = global_depth(n)
    seeds = g["seeds"]
    m = MDRPT(int(g["ntrees"]), td, 0.6, 2, n, n, d, seed=int(seeds[0]),
              local_seeds=seeds[1:], exact=True)
    m.grow_trees(X, 0.0, locality, int(g["nn"]))
    return m


@pytest.mark.gpu
def test_ubyte_60k_locality_leaves_and_edges_equal_reference(torch):
    g = _fixture("scale_c1_u8")
    X = _rows(g)
    m = _mdrpt(g, X, locality=True)
    assert m.gd == int(g["gd"]) and m.ld == int(g["ld"]) and m.n_final == int(g["n_final"])
    got = _leaf_shas(m.final_order.cpu().numpy(), m.final_offsets.cpu().numpy())
    assert got == list(g["leaf_sha256"])
    idx, dist = m.gather_nns(int(g["nn"]))
    res = _check_edges_up_to_ties(X, g["edge_ids"], idx.cpu().numpy(), dist.cpu().numpy())
    assert res["fail"] == 0, res
    assert res["tie"] <= 0.01 * X.shape[0], res


@pytest.mark.gpu
def test_fbin_131k_leaves_and_edges_equal_reference(torch):
    g = _fixture("scale_c2_f32")
    X = _rows(g)
    m = _mdrpt(g, X, locality=False)
    assert m.gd == int(g["gd"]) and m.ld == int(g["ld"]) and m.n_final == int(g["n_final"])
    got = _leaf_shas(m.final_order.cpu().numpy(), m.final_offsets.cpu().numpy())
    assert got == list(g["leaf_sha256"])
    idx, dist = m.gather_nns(int(g["nn"]))
    res = _check_edge_hash(g, idx.cpu().numpy(), dist.cpu().numpy())
    assert res["fail"] == 0, res
    # the single call gives the same lists
    i2, d2, _ = build_graph(X, int(g["ntrees"]), int(g["nn"]), int(g["seeds"][0]),
                            local_seeds=g["seeds"][1:])
    assert np.array_equal(i2, idx.cpu().numpy()) and d2.tobytes() == dist.cpu().numpy().tobytes()


@pytest.mark.gpu
def test_ubyte_60k_default_spread_is_an_error_status_where_the_reference_stops(torch):
    g = _fixture("scale_c1_u8")
    assert "length_error" in str(g["sigma20_reference_error"])
    X = synth.clustered_u8(60_000, 784, sigma_p=20.0, seed=1)
    with pytest.raises(DrptError) as e:
        build_graph(X, 8, 10, int(g["seeds"][0]), local_seeds=g["seeds"][1:], locality=True)
    assert e.value.status_name in ("DRPT_ERR_EMPTY_LEAF", "DRPT_ERR_DEPTH_OUT_OF_RANGE")
