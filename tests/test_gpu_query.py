"""Out-of-sample queries against a built index (drpt_index_build /
drpt_index_query): recall of held-out points against FP64 exact neighbours,
exact FP32 distances, indexed points finding themselves, learned trees, host
u8 queries and the argument checks.  Needs a B200."""
import numpy as np
import pytest

from drpt_b200 import DrptError, build_index, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as _t
    if not _t.cuda.is_available():
        pytest.skip("no CUDA device")
    return _t


def _exact(torch, X, Q, k):
    """FP64 exact k nearest rows of X for every row of Q: (idx, dist)."""
    Xd = torch.as_tensor(np.asarray(X, np.float64), device="cuda")
    Qd = torch.as_tensor(np.asarray(Q, np.float64), device="cuda")
    d2 = (Qd * Qd).sum(1)[:, None] + (Xd * Xd).sum(1)[None, :] - 2.0 * Qd @ Xd.T
    i = torch.topk(d2, k + 8, dim=1, largest=False).indices
    exact = torch.sqrt(((Xd[i] - Qd[:, None, :]) ** 2).sum(-1))
    o = torch.argsort(exact, dim=1, stable=True)[:, :k]
    return torch.gather(i, 1, o).cpu().numpy(), torch.gather(exact, 1, o).cpu().numpy()


def _recall(found, true):
    return np.mean([len(np.intersect1d(a, b)) / true.shape[1] for a, b in zip(found, true)])


@pytest.fixture(scope="module")
def clustered(torch):
    X = synth.clustered_f32(101_000, 128, n_clusters=100, seed=21)
    return X[:100_000], X[100_000:]


def test_held_out_queries(torch, clustered):
    X, Q = clustered
    Xd, Qd = torch.from_numpy(X).cuda(), torch.from_numpy(Q).cuda()
    index, _, _, _ = build_index(Xd, 6, 10, 7, leaf_size=1024)
    idx, dist = index.query(Qd, 10)
    torch.cuda.synchronize()
    I, D = idx.cpu().numpy(), dist.cpu().numpy()
    ti, _ = _exact(torch, X, Q, 10)
    assert _recall(I, ti) >= 0.85
    assert (I >= 0).all() and (I < len(X)).all()
    assert (D[:, 1:] >= D[:, :-1]).all()
    for q in range(0, len(Q), 97):
        assert len(np.unique(I[q])) == 10
        for j in (0, 5, 9):
            ref = np.sqrt(np.sum((X[I[q, j]].astype(np.float64) - Q[q]) ** 2))
            assert abs(D[q, j] - ref) <= 2e-6 * ref
    # the same queries from host memory give the same lists
    hi, hd = index.query(Q, 10)
    assert np.array_equal(hi, I) and np.array_equal(hd, D)
    index.close()


def test_indexed_points_find_themselves(torch, clustered):
    X, _ = clustered
    index, _, _, _ = build_index(torch.from_numpy(X).cuda(), 4, 10, 3, leaf_size=512)
    sel = np.arange(0, len(X), 997)
    idx, dist = index.query(X[sel], 5)
    assert (idx[:, 0] == sel).all() and (dist[:, 0] == 0).all()


def test_learned_index_and_u8(torch):
    X = synth.latent_manifold_f32(60_000, 256, seed=5)
    Q = synth.latent_manifold_f32(60_500, 256, seed=5)[60_000:]
    index, _, _, st = build_index(torch.from_numpy(X).cuda(), 8, 10, 1, leaf_size=1024,
                                  learned_trees=4, learn_sample=4096, learn_iters=5)
    assert st.ms_learn > 0
    idx, dist = index.query(Q, 10)
    ti, _ = _exact(torch, X, Q, 10)
    assert _recall(idx, ti) >= 0.6
    U = synth.clustered_u8(20_000, 784, seed=1)
    uindex, _, _, _ = build_index(U, 6, 10, 2, leaf_size=1024)
    ui, ud = uindex.query(U[:50], 10)
    assert (ui[:, 0] == np.arange(50)).all() and (ud[:, 0] == 0).all()


def test_query_argument_checks(torch, clustered):
    X, Q = clustered
    index, _, _, _ = build_index(X[:20_000], 2, 10, 1)
    with pytest.raises(DrptError) as e:
        index.query(Q, 33)
    assert e.value.status == 8
    with pytest.raises(DrptError) as e:
        index.query(Q[:, :64].copy(), 10)
    assert e.value.status == 1
    with pytest.raises(DrptError) as e:
        build_index(X[:20_000], 2, 10, 1, mode="exact")
    assert e.value.status == 1
