"""The autotuner and the list width on a B200: the tuner measures every
candidate, picks by the rule, caches, and its choice rebuilds to the same
graph; list widths outside 16 / 32 or below nn are rejected.  Needs a B200."""
import numpy as np
import pytest

from drpt_b200 import DrptError, autotune, build_graph, build_graph_batched, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as _t
    if not _t.cuda.is_available():
        pytest.skip("no CUDA device")
    return _t


def test_tune_batched_picks_and_caches(torch, tmp_path):
    sizes = [3000, 12000, 5000, 20000, 8000, 2500]
    sets = [synth.batch_dataset(m, 32, seed=50 + i) for i, m in enumerate(sizes)]
    offs = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    X = torch.from_numpy(np.concatenate(sets)).cuda()
    cache = str(tmp_path / "tune.json")
    r = autotune.tune_batched(X, offs, 6, 12, 3, leaf_sizes=(256, 512), reps=1,
                              queries_per_set=30, cache_path=cache)
    assert not r["cached"] and len(r["trials"]) == 4  # two leaf sizes x widths 16 and 32
    assert (r["leaf_size"], r["list_width"]) in {(t["leaf_size"], t["list_width"])
                                                  for t in r["trials"]}
    assert autotune.choose(r["trials"], 0.90)["ms"] == r["ms"]
    again = autotune.tune_batched(X, offs, 6, 12, 3, leaf_sizes=(256, 512), reps=1,
                                  queries_per_set=30, cache_path=cache)
    assert again["cached"] and again["leaf_size"] == r["leaf_size"]
    # the chosen setting rebuilds to the same graph outside the tuner
    i1, d1, _ = build_graph_batched(X, offs, 6, 12, 3, leaf_size=r["leaf_size"],
                                    list_width=r["list_width"])
    i2, d2, _ = build_graph_batched(X, offs, 6, 12, 3, leaf_size=r["leaf_size"],
                                    list_width=r["list_width"], use_graph=True)
    torch.cuda.synchronize()
    assert torch.equal(i1, i2) and torch.equal(d1, d2)


def test_list_width(torch):
    X = torch.from_numpy(synth.clustered_f32(40_000, 64, n_clusters=40, seed=9)).cuda()
    i16, d16, _ = build_graph(X, 4, 10, 5, mode="mixed", leaf_size=512, list_width=16)
    i0, d0, _ = build_graph(X, 4, 10, 5, mode="mixed", leaf_size=512)
    assert torch.equal(i16, i0) and torch.equal(d16, d0)  # 16 is the default for nn <= 10
    i32, d32, _ = build_graph(X, 4, 10, 5, mode="mixed", leaf_size=512, list_width=32)
    torch.cuda.synchronize()
    # more candidates can only bring nearer neighbours: the k-th distance never grows
    assert (d32[:, -1] <= d16[:, -1]).float().mean().item() > 0.99
    for bad in (24, 8):
        with pytest.raises(DrptError) as e:
            build_graph(X, 4, 10, 5, mode="mixed", leaf_size=512, list_width=bad)
        assert e.value.status == 1
    with pytest.raises(DrptError) as e:  # 16 keys cannot hold 20 neighbours
        build_graph(X, 4, 20, 5, mode="mixed", leaf_size=512, list_width=16)
    assert e.value.status == 1


def test_tune_graph_picks_a_measured_setting(torch):
    X = torch.from_numpy(synth.clustered_f32(60_000, 32, n_clusters=60, seed=8)).cuda()
    r = autotune.tune_graph(X, 4, 10, 2, leaf_sizes=(512, 1024), reps=1, queries=200)
    assert len(r["trials"]) == 4 and not r["cached"]
    assert autotune.choose(r["trials"], 0.90) == min(
        [t for t in r["trials"] if t["recall"] >= 0.90] or [max(r["trials"],
                                                               key=lambda t: t["recall"])],
        key=lambda t: t["ms"])
    i1, d1, _ = build_graph(X, 4, 10, 2, mode="mixed", leaf_size=r["leaf_size"],
                            list_width=r["list_width"])
    assert i1.shape == (60_000, 10) and (i1 >= 0).all()
