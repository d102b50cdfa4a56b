"""Parity of the CUDA path (through the C ABI) with the reference's golden
fixtures and with the CPU oracle.  Needs a B200."""
import glob
import os

import numpy as np
import pytest

import oracle
from drpt_b200 import MDRPT, DrptError, build_graph, global_depth
from tests import knn_compare
from tests.conftest import GOLDEN

pytestmark = pytest.mark.gpu

CASES = sorted(glob.glob(os.path.join(GOLDEN, "case_*.npz")))
OK_CASES = [c for c in CASES if "expect_error" not in np.load(c).files]
ERR_CASES = [c for c in CASES if "expect_error" in np.load(c).files]


def _id(path):
    return os.path.basename(path)[5:-4]


@pytest.fixture(scope="module")
def torch():
    import torch as _t
    if not _t.cuda.is_available():
        pytest.skip("no CUDA device")
    return _t


def _mdrpt(g, exact=True, locality=False):
    X = g["X"]
    n, d = X.shape
    T, nn = int(g["ntrees"]), int(g["nn"])
    td, _ = global_depth(n)
    m = MDRPT(T, td, 0.6, 2, n, n, d, seed=int(g["seeds"][0]), exact=exact)
    m.grow_trees(X, 0.0, locality, nn)
    return m


@pytest.mark.parametrize("case", OK_CASES, ids=_id)
def test_projection_bit_exact(torch, case):
    g = np.load(case)
    m = _mdrpt(g)
    assert np.array_equal(m.B, g["B"])
    T, gd = int(g["ntrees"]), int(g["gd"])
    P = m.P.cpu().numpy()  # (T*(gd-1)) x n
    want = g["P"] if g["P"].size else oracle.project(g["X"], g["B"])
    cols = [t * gd + lv for t in range(T) for lv in range(gd - 1)]
    assert P.tobytes() == np.ascontiguousarray(want[:, cols].T).tobytes()


@pytest.mark.parametrize("case", OK_CASES, ids=_id)
def test_global_trees_and_medians_bit_exact(torch, case):
    g = np.load(case)
    m = _mdrpt(g)
    T, gd = int(g["ntrees"]), int(g["gd"])
    P = oracle.project(g["X"], g["B"])
    order, offs, med = oracle.global_tree(P, T, gd)
    assert np.array_equal(m.global_offsets.cpu().numpy(), offs)
    assert np.array_equal(m.global_order.cpu().numpy(), order)
    got = m.medians.cpu().numpy().reshape(-1)[: med.size]
    assert got.tobytes() == med.reshape(-1).tobytes()


@pytest.mark.parametrize("case", OK_CASES, ids=_id)
def test_final_leaves_match_reference(torch, case):
    g = np.load(case)
    m = _mdrpt(g)
    assert m.ld == int(g["ld"]) and m.n_final == int(g["n_final"])
    assert np.array_equal(m.final_offsets.cpu().numpy(), g["final_offsets"])
    assert np.array_equal(m.final_order.cpu().numpy(), g["final_order"])


@pytest.mark.parametrize("case", OK_CASES, ids=_id)
def test_locality_final_leaves_match_reference(torch, case):
    """With the locality relabelling the final leaves come in the
    reference's -locality 1 order: leaf ids, not only the partition."""
    g = np.load(case)
    m = _mdrpt(g, locality=True)
    assert np.array_equal(m.final_offsets.cpu().numpy(), g["locality_final_offsets"])
    assert np.array_equal(m.final_order.cpu().numpy(), g["locality_final_order"])
    idx, dist = m.gather_nns(int(g["nn"]))
    m0 = _mdrpt(g)
    idx0, dist0 = m0.gather_nns(int(g["nn"]))
    assert np.array_equal(idx.cpu().numpy(), idx0.cpu().numpy())
    X = g["X"]
    i1, d1, _ = build_graph(X, int(g["ntrees"]), int(g["nn"]), int(g["seeds"][0]), locality=True)
    i2, d2, _ = build_graph(X, int(g["ntrees"]), int(g["nn"]), int(g["seeds"][0]))
    assert np.array_equal(i1, i2) and np.array_equal(d1, d2)


@pytest.mark.parametrize("case", OK_CASES, ids=_id)
def test_graph_matches_reference_up_to_ties(torch, case):
    g = np.load(case)
    X = g["X"]
    T, nn = int(g["ntrees"]), int(g["nn"])
    seeds = g["seeds"]
    idx, dist, st = build_graph(X, T, nn, int(seeds[0]), local_seeds=seeds[1:])
    assert st.global_depth == int(g["gd"]) and st.local_depth == int(g["ld"])
    ri, rd = knn_compare.reference_first_k(g["list_idx"], g["list_dist"], nn + 3)
    res = knn_compare.compare(ri[:, :nn], rd[:, :nn], idx.astype(np.int64), dist, rd)
    assert res["fail"] == 0, res
    if "ties" not in case:
        assert res["tie"] <= 0.01 * X.shape[0], res
    # the oracle orders ties the same way (distance, index): identical arrays
    o = oracle.build(X, T, nn, int(seeds[0]))
    assert np.array_equal(idx, o["knn_idx"])
    assert dist.tobytes() == o["knn_dist"].tobytes()


@pytest.mark.parametrize("case", OK_CASES[:2], ids=_id)
def test_mdrpt_interface_equals_single_call(torch, case):
    g = np.load(case)
    nn = int(g["nn"])
    m = _mdrpt(g)
    i1, d1 = m.gather_nns(nn)
    i2, d2, _ = build_graph(g["X"], int(g["ntrees"]), nn, int(g["seeds"][0]))
    assert np.array_equal(i1.cpu().numpy(), i2)
    assert np.array_equal(d1.cpu().numpy(), d2)


@pytest.mark.parametrize("case", ERR_CASES, ids=_id)
def test_reference_failures_become_statuses(torch, case):
    g = np.load(case)
    with pytest.raises(DrptError) as e:
        build_graph(g["X"], int(g["ntrees"]), int(g["nn"]), int(g["seeds"][0]))
    assert e.value.status in (2, 3)
    o = oracle.build(g["X"], int(g["ntrees"]), int(g["nn"]), int(g["seeds"][0]), want_knn=False)
    assert e.value.status == -o["status"]


def test_device_and_host_pointers_agree(torch):
    g = np.load(OK_CASES[0])
    X = g["X"]
    T, nn, s = int(g["ntrees"]), int(g["nn"]), int(g["seeds"][0])
    ih, dh, _ = build_graph(X, T, nn, s)
    Xd = torch.from_numpy(X).cuda()
    idv, ddv, _ = build_graph(Xd, T, nn, s)
    torch.cuda.synchronize()
    assert np.array_equal(ih, idv.cpu().numpy()) and np.array_equal(dh, ddv.cpu().numpy())


def _check_graph_properties(idx, dist, X, sample=200, seed=0):
    n, nn = idx.shape
    rows = np.arange(n)
    assert not (idx == rows[:, None]).any(), "self edge"
    valid = idx >= 0
    # sorted by (distance, index) and no duplicates
    d_ok = (dist[:, 1:] > dist[:, :-1]) | ((dist[:, 1:] == dist[:, :-1]) & (idx[:, 1:] > idx[:, :-1]))
    assert (d_ok | ~valid[:, 1:]).all()
    for p in np.random.default_rng(seed).choice(n, size=min(sample, n), replace=False):
        q = idx[p][idx[p] >= 0]
        assert len(np.unique(q)) == len(q)
        for j, qq in enumerate(q[:3]):
            assert dist[p, j] == oracle.distance(X[p].astype(np.float32), X[qq].astype(np.float32))


@pytest.mark.slow
def test_exact_bit_identical_to_oracle_medium(torch):
    from drpt_b200 import synth
    X = synth.clustered_f32(60_000, 48, n_clusters=300, seed=31)
    idx, dist, st = build_graph(X, 6, 10, 2024)
    o = oracle.build(X, 6, 10, 2024)
    assert np.array_equal(idx, o["knn_idx"])
    assert dist.tobytes() == o["knn_dist"].tobytes()


@pytest.mark.slow
def test_properties_at_scale(torch):
    """Config-2 distribution at 400k x 128 (16 trees): size-independent
    properties -- every tree's final leaves partition the points, lists are
    sorted, self-free and duplicate-free with bit-exact distances, and a
    second run is identical."""
    from drpt_b200 import synth
    X = synth.clustered_f32(400_000, 128, n_clusters=400, seed=32)
    Xd = torch.from_numpy(X).cuda()
    idx, dist, st = build_graph(Xd, 16, 10, 77)
    idx2, dist2, _ = build_graph(Xd, 16, 10, 77)
    torch.cuda.synchronize()
    assert torch.equal(idx, idx2) and torch.equal(dist, dist2)
    _check_graph_properties(idx.cpu().numpy(), dist.cpu().numpy(), X)
    td, gd = global_depth(len(X))
    m = MDRPT(16, td, 0.6, 2, len(X), len(X), 128, seed=77)
    m.grow_trees(Xd, 0.0, False, 10)
    fo = m.final_order.cpu().numpy()
    for t in range(16):
        assert np.array_equal(np.sort(fo[t]), np.arange(len(X)))


def test_fast_mode_is_a_valid_graph(torch):
    g = np.load(OK_CASES[1])
    X = g["X"]
    idx, dist, st = build_graph(X, int(g["ntrees"]), int(g["nn"]), int(g["seeds"][0]), mode="fast")
    _check_graph_properties(idx, dist, X.astype(np.float32))
    idx_e, _, _ = build_graph(X, int(g["ntrees"]), int(g["nn"]), int(g["seeds"][0]))
    q = np.random.default_rng(0).choice(len(X), 500, replace=False)
    ti, _ = oracle.exact_knn(X.astype(np.float32), q, int(g["nn"]))
    r_fast = oracle.recall_at_k(idx[q], ti)
    r_exact = oracle.recall_at_k(idx_e[q], ti)
    assert abs(r_fast - r_exact) < 0.1, (r_fast, r_exact)
