"""The tree-sharded build's exchange (drpt_b200.shard) with two gloo ranks on
the CPU: each rank's lists come from the CPU oracle for its share of the
trees, the exchange and merge must give every rank exactly what merging all
ranks' lists in one process gives.  The GPU path differs only in where the
lists come from (build_graph) and in the merge kernel."""
import multiprocessing as mp
import socket
from datetime import timedelta

import numpy as np
import pytest

import oracle
from drpt_b200 import synth
from drpt_b200.shard import exchange_merge, rank_seed, row_bounds, tree_share


def _np_merge(li, ld, k):
    """Nearest distinct candidates by (distance, index), -1 / +inf padded."""
    import torch
    li, ld = li.numpy(), ld.numpy()
    rows = li.shape[0]
    oi = np.full((rows, k), -1, np.int32)
    od = np.full((rows, k), np.inf, np.float32)
    for p in range(rows):
        ii, dd = li[p].reshape(-1), ld[p].reshape(-1)
        keep = ii >= 0
        ii, dd = ii[keep], dd[keep]
        seen, w = set(), 0
        for j in np.lexsort((ii, dd)):
            if int(ii[j]) in seen:
                continue
            seen.add(int(ii[j]))
            oi[p, w], od[p, w] = ii[j], dd[j]
            w += 1
            if w == k:
                break
    return torch.from_numpy(oi), torch.from_numpy(od)


def _rank_lists(X, ntrees, nn, seed, world, rank):
    share = tree_share(ntrees, world, rank)
    n = X.shape[0]
    if share == 0:
        return np.full((n, nn), -1, np.int32), np.full((n, nn), np.inf, np.float32)
    r = oracle.build(X, share, nn, rank_seed(seed, rank))
    assert r["status"] == 0
    return r["knn_idx"].astype(np.int32), r["knn_dist"].astype(np.float32)


def _worker(rank, world, port, X, ntrees, nn, seed, gather, q):
    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=timedelta(seconds=120))
    try:
        li, ld = _rank_lists(X, ntrees, nn, seed, world, rank)
        oi, od, bounds = exchange_merge(torch.from_numpy(li), torch.from_numpy(ld), nn,
                                        merge=_np_merge, gather=gather)
        q.put((rank, oi.numpy(), od.numpy(), bounds))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run(X, ntrees, nn, seed, world, gather):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, X, ntrees, nn, seed, gather, q))
             for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(world):
        rank, oi, od, bounds = q.get(timeout=300)
        out[rank] = (oi, od, bounds)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return out


@pytest.mark.parametrize("ntrees,gather", [(3, True), (1, True), (3, False)])
def test_exchange_equals_single_process_merge(ntrees, gather):
    X = synth.clustered_f32(3001, 24, n_clusters=30, seed=5)
    nn, seed, world = 6, 4242, 2
    lists = [_rank_lists(X, ntrees, nn, seed, world, r) for r in range(world)]
    import torch
    li = torch.from_numpy(np.stack([l[0] for l in lists], axis=1))
    ld = torch.from_numpy(np.stack([l[1] for l in lists], axis=1))
    want_i, want_d = (t.numpy() for t in _np_merge(li, ld, nn))
    out = _run(X, ntrees, nn, seed, world, gather)
    bounds = row_bounds(len(X), world)
    for r in range(world):
        oi, od, b = out[r]
        assert b == bounds
        lo, hi = (0, len(X)) if gather else (bounds[r], bounds[r + 1])
        assert np.array_equal(oi, want_i[lo:hi]) and np.array_equal(od, want_d[lo:hi])
    # every rank's trees contributed: the merged lists are at least as near as
    # rank 0's own lists, entry by entry
    assert (want_d[:, 0] <= lists[0][1][:, 0]).all()


def test_tree_shares_and_seeds():
    assert [tree_share(6, 4, r) for r in range(4)] == [2, 2, 1, 1]
    assert sum(tree_share(13, 8, r) for r in range(8)) == 13
    assert rank_seed(77, 0) == 77 and len({rank_seed(77, r) for r in range(8)}) == 8
    assert row_bounds(10, 3) == [0, 3, 6, 10]
