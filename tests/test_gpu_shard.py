"""The tree-sharded build on one B200: the library's merge kernel follows the
merge rule the CPU exchange test uses, and a one-rank NCCL group gives the
single-GPU graph.  (Runs of two or more GPUs are not available here; the
exchange itself is covered by the gloo test on the CPU.)  Needs a B200."""
import socket

import numpy as np
import pytest

from drpt_b200 import build_graph, synth
from drpt_b200.shard import build_graph_sharded, device_merge, rank_seed
from tests.test_shard import _np_merge

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as _t
    if not _t.cuda.is_available():
        pytest.skip("no CUDA device")
    return _t


def test_device_merge_follows_the_rule(torch):
    X = torch.from_numpy(synth.clustered_f32(60_000, 64, n_clusters=60, seed=3)).cuda()
    lists = [build_graph(X, 2, 10, rank_seed(7, r), mode="mixed", leaf_size=512)[:2]
             for r in range(3)]
    li = torch.stack([l[0] for l in lists], dim=1)
    ld = torch.stack([l[1] for l in lists], dim=1)
    mi, md = device_merge(li, ld, 10)
    torch.cuda.synchronize()
    rows = slice(0, 60_000, 7)
    wi, wd = _np_merge(li[rows].cpu(), ld[rows].cpu(), 10)
    assert np.array_equal(mi[rows].cpu().numpy(), wi.numpy())
    assert np.array_equal(md[rows].cpu().numpy(), wd.numpy())


def test_one_rank_group_gives_the_single_gpu_graph(torch):
    import torch.distributed as dist
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1)
    try:
        X = torch.from_numpy(synth.clustered_f32(50_000, 32, n_clusters=50, seed=4)).cuda()
        si, sd, bounds = build_graph_sharded(X, 4, 10, 11, mode="mixed", leaf_size=512)
        ri, rd, _ = build_graph(X, 4, 10, 11, mode="mixed", leaf_size=512)
        torch.cuda.synchronize()
        assert bounds == [0, 50_000]
        assert torch.equal(si, ri) and torch.equal(sd, rd)
    finally:
        dist.destroy_process_group()
