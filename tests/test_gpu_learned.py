"""Learned splits: the GPU training kernels' loss and gradient against the CPU
FP64 oracle (oracle/learned.py), the recall the learned trees gain over
random-projection trees at equal tree count on the latent-manifold workload,
determinism and the argument checks.  Needs a B200."""
import ctypes

import numpy as np
import pytest

from drpt_b200 import DrptError, _lib, build_graph, recall, synth
from oracle import learned

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as _t
    if not _t.cuda.is_available():
        pytest.skip("no CUDA device")
    return _t


def _gpu_grad(X, params, node, nbr):
    S, d = X.shape
    grad = np.zeros_like(params)
    loss = ctypes.c_float()
    L = _lib.load()
    ctx = _lib.context(0)
    _lib.check(L.drpt_learn_gradient(ctx.handle, X.ctypes.data, S, d, params.ctypes.data,
                                     node.ctypes.data, nbr.ctypes.data, nbr.shape[1],
                                     grad.ctypes.data, ctypes.byref(loss)))
    return loss.value, grad


@pytest.mark.parametrize("S,d,k,nodes", [(600, 32, 5, 3), (2000, 96, 10, 8), (333, 256, 7, 1)])
def test_training_gradient_matches_oracle(torch, S, d, k, nodes):
    """One forward + backward of the split MLP on the GPU (FP32, BF16
    weights) against the FP64 oracle: loss within 1e-5 relative, every
    gradient entry within 1e-4 of the largest."""
    rng = np.random.default_rng(S + d)
    X = rng.standard_normal((S, d)).astype(np.float32)
    node = rng.integers(0, nodes, size=S).astype(np.int32)
    nbr = rng.integers(0, S, size=(S, k)).astype(np.int32)
    nbr[rng.random((S, k)) < 0.05] = -1
    W1 = (rng.standard_normal((learned.HIDDEN, d)) / np.sqrt(d)).astype(np.float32)
    b1 = (rng.standard_normal(learned.HIDDEN) * 0.1).astype(np.float32)
    w2 = (rng.standard_normal(learned.HIDDEN) / 8).astype(np.float32)
    b2 = np.float32(-0.3)
    params = np.concatenate([W1.ravel(), b1, w2, [b2]]).astype(np.float32)
    loss, grad = _gpu_grad(X, params, node, nbr)
    L, dW1, db1, dw2, db2 = learned.loss_and_grad(X, W1, b1, w2, b2, node, nbr)
    want = np.concatenate([dW1.ravel(), db1, dw2, [db2]])
    assert abs(loss - L) <= 1e-5 * abs(L)
    assert np.abs(grad - want).max() <= 1e-4 * np.abs(want).max()


@pytest.fixture(scope="module")
def manifold(torch):
    X = synth.latent_manifold_f32(100_000, 256, seed=5)
    Xd = torch.from_numpy(X).cuda()
    q = recall.sample_queries(len(X), 400, seed=9)
    ti, _ = recall.exact_knn_fp64(Xd, q, 10)
    return X, Xd, q, ti


def test_learned_trees_gain_over_random_trees(torch, manifold):
    """At equal tree count the trained splits beat random projections on the
    16-dimensional manifold, and training lowers the split loss."""
    X, Xd, q, ti = manifold
    rec = {}
    for learned_trees in (0, 4, 8):
        idx, _, st = build_graph(Xd, 8, 10, 12345, mode="mixed", leaf_size=1024,
                                 learned_trees=learned_trees)
        rec[learned_trees] = recall.recall_at_k(idx.cpu().numpy()[q], ti)
        if learned_trees:
            assert st.learn_loss_end < 0.8 * st.learn_loss_start, st.as_dict()
            assert st.ms_learn > 0
    assert rec[4] >= rec[0] + 0.04, rec
    assert rec[8] >= rec[0] + 0.08, rec


def test_learned_build_is_deterministic(torch, manifold):
    _, Xd, _, _ = manifold
    a = build_graph(Xd, 6, 10, 3, mode="mixed", leaf_size=1024, learned_trees=3,
                    learn_sample=4096, learn_iters=5)
    b = build_graph(Xd, 6, 10, 3, mode="mixed", leaf_size=1024, learned_trees=3,
                    learn_sample=4096, learn_iters=5)
    torch.cuda.synchronize()
    assert torch.equal(a[0], b[0]) and torch.equal(a[1], b[1])


def test_learned_argument_checks(torch):
    X = np.random.default_rng(0).random((5000, 64), dtype=np.float32)
    with pytest.raises(DrptError) as e:
        build_graph(X, 2, 10, 1, mode="mixed", learned_trees=3)
    assert e.value.status == 1
    X = np.random.default_rng(0).random((5000, 320), dtype=np.float32)
    with pytest.raises(DrptError) as e:
        build_graph(X, 2, 10, 1, mode="mixed", learned_trees=1)
    assert e.value.status == 8


def test_large_sample_trains_in_chunks(torch, manifold):
    """A sample above the leaf kernel's 8,192-point limit finds its
    neighbour pairs in chunks; training still lowers the loss, the build is
    deterministic and keeps the gain over random trees; samples beyond
    2^20 are rejected."""
    X, Xd, q, ti = manifold
    a = build_graph(Xd, 8, 10, 12345, mode="mixed", leaf_size=1024, learned_trees=8,
                    learn_sample=30_000)
    b = build_graph(Xd, 8, 10, 12345, mode="mixed", leaf_size=1024, learned_trees=8,
                    learn_sample=30_000)
    torch.cuda.synchronize()
    assert torch.equal(a[0], b[0])
    st = a[2]
    assert st.learn_loss_end < 0.8 * st.learn_loss_start, st.as_dict()
    r0, _, _ = build_graph(Xd, 8, 10, 12345, mode="mixed", leaf_size=1024)
    assert (recall.recall_at_k(a[0].cpu().numpy()[q], ti)
            >= recall.recall_at_k(r0.cpu().numpy()[q], ti) + 0.08)
    with pytest.raises(DrptError) as e:
        build_graph(Xd, 4, 10, 1, mode="mixed", learned_trees=2, learn_sample=(1 << 20) + 1)
    assert e.value.status == 1
