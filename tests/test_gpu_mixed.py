"""The mixed-precision form (BF16 tcgen05 leaf tiles, FP32 re-rank, FP64
boundary check): recall against FP64 exact neighbours, exact FP32 output
distances, determinism and its stated limits.  Needs a B200."""
import numpy as np
import pytest

import oracle
from drpt_b200 import DrptError, build_graph, recall, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as _t
    if not _t.cuda.is_available():
        pytest.skip("no CUDA device")
    return _t


def _exact_fp32(a, b):
    return oracle.distance(a.astype(np.float32), b.astype(np.float32))


def _close(got, a, b, rtol=2e-6):
    """The mixed form's distances are FP32 sums in a fixed pairwise order; they
    agree with the FP64 distance to a few units in the last place."""
    ref = float(np.sqrt(np.sum((a.astype(np.float64) - b.astype(np.float64)) ** 2)))
    return abs(float(got) - ref) <= rtol * max(ref, 1e-30)


@pytest.fixture(scope="module")
def clustered(torch):
    X = synth.clustered_f32(120_000, 128, n_clusters=120, seed=41)
    return X, torch.from_numpy(X).cuda()


def test_mixed_recall_and_distances(torch, clustered):
    X, Xd = clustered
    idx, dist, st = build_graph(Xd, 6, 10, 99, mode="mixed", leaf_size=1024)
    torch.cuda.synchronize()
    I, D = idx.cpu().numpy(), dist.cpu().numpy()
    q = recall.sample_queries(len(X), 400, seed=3)
    ti, _ = recall.exact_knn_fp64(Xd, q, 10)
    r = recall.recall_at_k(I[q], ti)
    assert r >= 0.85, r
    assert not (I == np.arange(len(X))[:, None]).any()
    assert (I >= 0).all()
    assert ((D[:, 1:] >= D[:, :-1])).all()
    for p in q[:25]:
        assert len(np.unique(I[p])) == I.shape[1]
        for j in range(0, 10, 3):
            assert _close(D[p, j], X[p], X[I[p, j]])


def test_mixed_is_deterministic(torch, clustered):
    _, Xd = clustered
    a = build_graph(Xd, 4, 10, 5, mode="mixed", leaf_size=512)
    b = build_graph(Xd, 4, 10, 5, mode="mixed", leaf_size=512)
    torch.cuda.synchronize()
    assert torch.equal(a[0], b[0]) and torch.equal(a[1], b[1])


def test_mixed_recall_grows_with_trees(torch, clustered):
    X, Xd = clustered
    q = recall.sample_queries(len(X), 300, seed=4)
    ti, _ = recall.exact_knn_fp64(Xd, q, 10)
    rs = []
    for T in (1, 3, 6):
        idx, _, _ = build_graph(Xd, T, 10, 11, mode="mixed", leaf_size=1024)
        rs.append(recall.recall_at_k(idx.cpu().numpy()[q], ti))
    assert rs[0] < rs[1] <= rs[2] + 1e-9, rs


def test_mixed_u8_and_k16(torch):
    X = synth.clustered_u8(30_000, 784 // 7 * 2, seed=8)  # 224 dims, u8
    Xd = torch.from_numpy(X).cuda()
    idx, dist, _ = build_graph(Xd, 4, 16, 3, mode="mixed", leaf_size=1024)
    torch.cuda.synchronize()
    I, D = idx.cpu().numpy(), dist.cpu().numpy()
    for p in (0, 17, 2999):
        assert _close(D[p, 0], X[p], X[I[p, 0]])
    q = recall.sample_queries(len(X), 200, seed=5)
    ti, _ = recall.exact_knn_fp64(Xd, q, 16)
    assert recall.recall_at_k(I[q], ti) > 0.5


def test_mixed_limits_are_reported(torch):
    # d above 1,024 or not a multiple of 4, nn above 32: DRPT_ERR_UNSUPPORTED
    for d, nn in [(1028, 10), (962, 10), (64, 33)]:
        X = np.random.default_rng(0).random((5000, d), dtype=np.float32)
        with pytest.raises(DrptError) as e:
            build_graph(X, 2, nn, 1, mode="mixed")
        assert e.value.status == 8, (d, nn)
    X = np.random.default_rng(0).random((5000, 64), dtype=np.float32)
    with pytest.raises(DrptError) as e:
        build_graph(X, 2, 10, 1, mode="mixed", precision="bf16", leaf_size=-5)
    assert e.value.status == 1  # DRPT_ERR_INVALID_ARG


def test_mixed_matches_its_fp32_counterpart(torch, clustered):
    """Same trees and leaves: the FP32 whole-leaf form returns the exact k
    best of the candidate set; the mixed form (BF16 ranking, FP32 re-rank)
    can only miss a few of them and never returns a closer list."""
    X, Xd = clustered
    im, dm, _ = build_graph(Xd, 4, 10, 21, mode="mixed", leaf_size=1024)
    i3, d3, _ = build_graph(Xd, 4, 10, 21, mode="fp32_leaf", leaf_size=1024)
    torch.cuda.synchronize()
    im, dm, i3, d3 = (t.cpu().numpy() for t in (im, dm, i3, d3))
    assert (d3 <= dm * (1 + 2e-6)).all()        # exact k best of the same candidates
    same = np.mean([len(np.intersect1d(a, b)) / 10.0 for a, b in zip(im, i3)])
    assert same >= 0.99, same
    for p in (0, 5, 999):
        assert d3[p, 0] == _exact_fp32(X[p], X[i3[p, 0]])


def _recall(idx, q, ti):
    return recall.recall_at_k(idx.cpu().numpy()[q], ti)


def test_mixed_wide_rows_bf16_and_fp8(torch):
    """d = 960 streams the operand K blocks through shared memory; nn = 20
    keeps 32 candidates per point.  With the same trees the tensor-core forms
    find what the exact FP32 whole-leaf form finds, in BF16 and in E4M3 with
    per-row scales, and their output distances are FP32 distances."""
    X = synth.anisotropic_f32(60_000, 960, n_clusters=15, seed=3)
    Xd = torch.from_numpy(X).cuda()
    q = recall.sample_queries(len(X), 200, seed=6)
    ti, _ = recall.exact_knn_fp64(Xd, q, 20)
    i3, d3, _ = build_graph(Xd, 4, 20, 7, mode="fp32_leaf", leaf_size=1024)
    r3 = _recall(i3, q, ti)
    d3 = d3.cpu().numpy()
    for prec in ("bf16", "fp8"):
        im, dm, _ = build_graph(Xd, 4, 20, 7, mode="mixed", leaf_size=1024, precision=prec)
        torch.cuda.synchronize()
        rm = _recall(im, q, ti)
        assert rm >= r3 - 0.02, (prec, rm, r3)
        I, D = im.cpu().numpy(), dm.cpu().numpy()
        assert (d3 <= D * (1 + 2e-6)).all(), prec
        same = np.mean([len(np.intersect1d(a, b)) / 20.0 for a, b in zip(I, i3.cpu().numpy())])
        assert same >= 0.97, (prec, same)
        for p in q[:10]:
            for j in (0, 9, 19):
                assert _close(D[p, j], X[p], X[I[p, j]]), (prec, p, j)


def test_mixed_mnist_shaped_u8(torch):
    """60,000 x 784 u8 (IDX3-shaped): 8 trees of whole leaves reach recall@10
    0.85 in BF16 and in FP8."""
    X = synth.clustered_u8(60_000, 784, seed=1)
    Xd = torch.from_numpy(X).cuda()
    q = recall.sample_queries(len(X), 300, seed=7)
    ti, _ = recall.exact_knn_fp64(Xd, q, 10)
    for prec in ("bf16", "fp8"):
        idx, _, _ = build_graph(Xd, 8, 10, 12345, mode="mixed", leaf_size=1024, precision=prec)
        assert _recall(idx, q, ti) >= 0.85, prec


def test_mixed_fp8_low_dimension(torch, clustered):
    """E4M3 at d = 128: coarser ranking than BF16, still recall@10 >= 0.85
    with 6 trees, and the FP32 re-rank keeps the output distances exact."""
    X, Xd = clustered
    q = recall.sample_queries(len(X), 300, seed=8)
    ti, _ = recall.exact_knn_fp64(Xd, q, 10)
    idx, dist, _ = build_graph(Xd, 6, 10, 99, mode="mixed", leaf_size=1024, precision="fp8")
    assert _recall(idx, q, ti) >= 0.85
    I, D = idx.cpu().numpy(), dist.cpu().numpy()
    for p in q[:10]:
        assert _close(D[p, 0], X[p], X[I[p, 0]])


def test_fp32_gram_form_matches_the_fp32_whole_leaf_recall(torch, clustered):
    """The FP32 CUDA-core Gram form (||y||^2 - 2 x.y by FFMA, re-ranked in
    exact FP32) on the mixed form's trees: recall within 0.005 of the same
    trees brute-forced with the exact per-pair FP32 distance, FP32 output
    distances, no self and no duplicates."""
    X, Xd = clustered
    q = recall.sample_queries(len(X), 400, seed=3)
    ti, _ = recall.exact_knn_fp64(Xd, q, 10)
    gi, gd, _ = build_graph(Xd, 6, 10, 99, mode="fp32_gram", leaf_size=1024)
    li, _, _ = build_graph(Xd, 6, 10, 99, mode="fp32_leaf", leaf_size=1024)
    torch.cuda.synchronize()
    G, D, Lx = gi.cpu().numpy(), gd.cpu().numpy(), li.cpu().numpy()
    rg, rl = recall.recall_at_k(G[q], ti), recall.recall_at_k(Lx[q], ti)
    assert abs(rg - rl) <= 0.005, (rg, rl)
    assert not (G == np.arange(len(X))[:, None]).any() and (G >= 0).all()
    assert ((D[:, 1:] >= D[:, :-1])).all()
    for p in q[:25]:
        assert len(np.unique(G[p])) == G.shape[1]
        for j in range(0, 10, 3):
            assert _close(D[p, j], X[p], X[G[p, j]])
    # u8 rows (784 dimensions) and 32 candidates per tree
    U = synth.clustered_u8(8_000, 784, sigma_p=40.0, seed=7)
    ui, ud, _ = build_graph(U, 3, 16, 5, mode="fp32_gram", leaf_size=512)
    qu = np.arange(0, len(U), 97)
    tu, _ = oracle.exact_knn(U, qu, 16)
    assert recall.recall_at_k(ui[qu], tu) >= 0.8
    for p in qu[:10]:
        assert _close(ud[p, 0], U[p], U[ui[p, 0]])
