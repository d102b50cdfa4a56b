"""The CPU oracle against the golden fixtures produced by the reference
itself (tests/golden/make_golden.py).  No GPU."""
import glob
import os

import numpy as np
import pytest

import oracle
from tests import knn_compare
from tests.conftest import GOLDEN

CASES = sorted(glob.glob(os.path.join(GOLDEN, "case_*.npz")))
OK_CASES = [c for c in CASES if "expect_error" not in np.load(c).files]
ERR_CASES = [c for c in CASES if "expect_error" in np.load(c).files]


def _id(path):
    return os.path.basename(path)[5:-4]


def test_median_cases_bit_exact():
    g = np.load(os.path.join(GOLDEN, "median_cases.npz"))
    off = 0
    for i, sz in enumerate(g["sizes"]):
        vals = g["values"][off:off + sz]
        off += sz
        out4, _, _ = oracle.node_median(vals)
        for got, want, what in ((out4[0], g["mean"][i], "mean"), (out4[1], g["var"][i], "var"),
                                (out4[3], g["median"][i], "median")):
            assert (np.isnan(got) and np.isnan(want)) or \
                np.float32(got).tobytes() == np.float32(want).tobytes(), (i, what, got, want)


@pytest.mark.parametrize("case", OK_CASES, ids=_id)
def test_projection_matrix_and_P(case):
    g = np.load(case)
    d = g["X"].shape[1]
    L = int(g["gd"]) * int(g["ntrees"])
    B = oracle.projection_matrix(int(g["seeds"][0]), d, L, float(g["density"]))
    assert np.array_equal(B, g["B"])
    if g["P"].size:
        P = oracle.project(g["X"], B)
        assert P.tobytes() == g["P"].tobytes()


@pytest.mark.parametrize("case", OK_CASES, ids=_id)
def test_tree_assignment_and_lists(case):
    g = np.load(case)
    X = g["X"]
    T, nn = int(g["ntrees"]), int(g["nn"])
    seeds = g["seeds"]
    o = oracle.build(X, T, nn, int(seeds[0]), local_seeds=seeds[1:])
    assert o["status"] == 0
    assert o["info"].global_depth == int(g["gd"]) and o["info"].local_depth == int(g["ld"])
    assert np.array_equal(o["final_offsets"], g["final_offsets"])
    assert np.array_equal(o["final_order"], g["final_order"])
    ri, rd = knn_compare.reference_first_k(g["list_idx"], g["list_dist"], nn + 3)
    res = knn_compare.compare(ri[:, :nn], rd[:, :nn], o["knn_idx"], o["knn_dist"], rd)
    assert res["fail"] == 0, res
    assert res["exact"] + res["tie"] == X.shape[0]
    if "ties" not in case:
        assert res["tie"] <= 0.01 * X.shape[0], res


@pytest.mark.parametrize("case", ERR_CASES, ids=_id)
def test_reference_error_cases(case):
    g = np.load(case)
    o = oracle.build(g["X"], int(g["ntrees"]), int(g["nn"]), int(g["seeds"][0]), want_knn=False)
    # the reference throws std::out_of_range; the oracle reports depth (-2) or empty leaf (-3)
    assert o["status"] in (-2, -3)


@pytest.mark.parametrize("n,ld", [(1, 0), (2, 1), (7, 1), (100, 3), (1953, 5), (4099, 6)])
def test_local_perm_is_permutation(n, ld):
    if ld == 0:
        with pytest.raises(RuntimeError):
            oracle.local_perm(n, 1)
        return
    perm, first = oracle.local_perm(n, ld)
    assert sorted(perm.tolist()) == list(range(n))
    sizes = np.diff(first)
    assert first[0] == 0 and first[-1] == n and len(sizes) == 1 << ld
    assert sizes.max() - sizes.min() <= 1
