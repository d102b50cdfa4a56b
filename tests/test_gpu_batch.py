"""Batched builds (drpt_build_graph_batched): many independent datasets of
uneven sizes in one call, each dataset's graph identical to its own single
build, CUDA-graph replay, and the argument checks.  Needs a B200."""
import numpy as np
import pytest

from drpt_b200 import DrptError, build_graph, build_graph_batched, recall, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as _t
    if not _t.cuda.is_available():
        pytest.skip("no CUDA device")
    return _t


@pytest.fixture(scope="module")
def batch():
    """13 datasets of the batched workload's distribution (d = 96, 20-200
    Gaussians each), sizes log-uniform in [2,000, 40,000]."""
    sizes = synth.batch_sizes(13, 2_000, 40_000, seed=11)
    sets = [synth.batch_dataset(int(m), 96, seed=100 + i) for i, m in enumerate(sizes)]
    offs = np.concatenate([[0], np.cumsum([len(x) for x in sets])]).astype(np.int64)
    return sets, np.concatenate(sets), offs


@pytest.mark.parametrize("mode,precision", [("mixed", "bf16"), ("mixed", "fp8"),
                                            ("fp32_leaf", "bf16")])
def test_batch_equals_single_builds(torch, batch, mode, precision):
    sets, X, offs = batch
    Xd = torch.from_numpy(X).cuda()
    idx, dist, st = build_graph_batched(Xd, offs, 8, 16, 77, mode=mode, precision=precision,
                                        leaf_size=512)
    torch.cuda.synchronize()
    I, D = idx.cpu().numpy(), dist.cpu().numpy()
    for s, x in enumerate(sets):
        i1, d1, _ = build_graph(torch.from_numpy(x).cuda(), 8, 16, 77, mode=mode,
                                precision=precision, leaf_size=512)
        torch.cuda.synchronize()
        a, b = offs[s], offs[s + 1]
        assert np.array_equal(I[a:b], i1.cpu().numpy()), s
        assert D[a:b].tobytes() == d1.cpu().numpy().tobytes(), s


def test_batch_recall_and_host_pointers(torch, batch):
    sets, X, offs = batch
    idx, dist, _ = build_graph_batched(X, offs, 8, 16, 5, leaf_size=512)  # host in, host out
    for s in (0, 5, 12):
        x = sets[s]
        q = recall.sample_queries(len(x), 100, seed=s)
        ti, _ = recall.exact_knn_fp64(x, q, 16)
        got = idx[offs[s]:offs[s + 1]]
        assert (got >= 0).all() and (got < len(x)).all()
        assert recall.recall_at_k(got[q], ti) >= 0.9, s


def test_batch_graph_replay(torch, batch):
    _, X, offs = batch
    Xd = torch.from_numpy(X).cuda()
    idx = torch.empty((len(X), 16), dtype=torch.int32, device="cuda")
    dist = torch.empty((len(X), 16), dtype=torch.float32, device="cuda")
    want = build_graph_batched(Xd, offs, 8, 16, 3, leaf_size=512)
    torch.cuda.synchronize()
    for _ in range(3):  # eager + capture, then two replays
        idx.fill_(-7)
        build_graph_batched(Xd, offs, 8, 16, 3, leaf_size=512, use_graph=True, out=(idx, dist))
        torch.cuda.synchronize()
        assert torch.equal(idx, want[0]) and torch.equal(dist, want[1])
    # the replay reads the input again: new values in the same tensor
    Xd.mul_(1.5)
    want2 = build_graph_batched(Xd.clone(), offs, 8, 16, 3, leaf_size=512)
    build_graph_batched(Xd, offs, 8, 16, 3, leaf_size=512, use_graph=True, out=(idx, dist))
    torch.cuda.synchronize()
    assert torch.equal(idx, want2[0]) and torch.equal(dist, want2[1])


def test_batch_argument_checks(torch, batch):
    _, X, offs = batch
    with pytest.raises(DrptError) as e:
        build_graph_batched(X, offs + 1, 4, 10, 1)  # offsets[0] != 0 (and the end mismatches)
    assert e.value.status == 1
    bad = offs.copy()
    bad[1] = 1  # a one-row dataset
    with pytest.raises(DrptError) as e:
        build_graph_batched(X, bad, 4, 10, 1)
    assert e.value.status == 1
    with pytest.raises(DrptError) as e:
        build_graph_batched(X, offs, 4, 10, 1, use_graph=True)  # host pointers
    assert e.value.status == 1
