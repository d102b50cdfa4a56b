"""Tree-sharded k-NN graph over the ranks of a torch.distributed process
group: one process per GPU, the dataset replicated in every GPU's memory.

The reference spreads points and leaves over MPI ranks and exchanges leaf
data with Alltoallv (mdrpt.cpp:214-801).  Here the unit of work is the tree:
rank r builds `tree_share(T, G, r)` trees of its own (projection seed
`rank_seed(seed, r)`) over the whole dataset, which yields every point's
nearest neighbours among its leaf-mates in those trees.  One exchange step
remains: an all-to-all sends each point's list to the rank that owns the
point's range of rows, which merges the G lists into the point's k nearest
distinct candidates (the library's cross-tree merge kernel on the GPU); an
optional all-gather gives every rank the whole graph.

Bytes crossing NVLink per rank: n * k * 8 * (G - 1) / G for the exchange,
the same again for the all-gather.
"""
from __future__ import annotations

from . import _lib
from .graph import _is_cuda_tensor, _torch, build_graph


def tree_share(ntrees: int, world: int, rank: int) -> int:
    """Trees rank `rank` builds: the T trees dealt out as evenly as possible."""
    return ntrees // world + (1 if rank < ntrees % world else 0)


def rank_seed(seed: int, rank: int) -> int:
    """Projection seed of rank `rank`'s trees (rank 0 keeps `seed`)."""
    return (int(seed) + 0x9E3779B9 * int(rank)) & 0xFFFFFFFF


def row_bounds(n: int, world: int) -> list[int]:
    """Rows [bounds[r], bounds[r + 1]) are owned by rank r."""
    return [r * n // world for r in range(world + 1)]


def device_merge(lists_idx, lists_dist, k: int):
    """(rows, L, k) candidate lists per row on the GPU -> (rows, k) nearest
    distinct candidates by (distance, index), through the library's merge
    kernel (drpt_merge_candidates)."""
    torch = _torch()
    rows, L = int(lists_idx.shape[0]), int(lists_idx.shape[1])
    dev = lists_idx.device
    out_i = torch.empty((rows, k), dtype=torch.int32, device=dev)
    out_d = torch.empty((rows, k), dtype=torch.float32, device=dev)
    if rows == 0:
        return out_i, out_d
    ctx = _lib.context(dev.index or 0)
    s = torch.cuda.current_stream(dev).cuda_stream
    _lib.check(_lib.load().drpt_merge_candidates(
        ctx.handle, lists_idx.contiguous().data_ptr(), lists_dist.contiguous().data_ptr(), rows, L,
        k, out_i.data_ptr(), out_d.data_ptr(), s))
    return out_i, out_d


def exchange_merge(idx, dist, k: int, group=None, merge=device_merge, gather: bool = True):
    """idx / dist: this rank's (n, k) lists (int32 / float32 tensors on the
    group's device).  Each rank receives every rank's lists for the rows it
    owns, merges them with `merge` and, with `gather`, all ranks receive all
    rows.  Returns (idx, dist, bounds): the whole graph, or this rank's rows
    [bounds[rank], bounds[rank + 1])."""
    torch = _torch()
    import torch.distributed as dist_

    world = dist_.get_world_size(group)
    rank = dist_.get_rank(group)
    n = int(idx.shape[0])
    bounds = row_bounds(n, world)
    counts = [bounds[r + 1] - bounds[r] for r in range(world)]
    mine = counts[rank]
    recv_i = torch.empty(world * mine * k, dtype=idx.dtype, device=idx.device)
    recv_d = torch.empty(world * mine * k, dtype=dist.dtype, device=dist.device)
    splits_in = [c * k for c in counts]
    splits_out = [mine * k] * world
    dist_.all_to_all_single(recv_i, idx.contiguous().view(-1), splits_out, splits_in, group=group)
    dist_.all_to_all_single(recv_d, dist.contiguous().view(-1), splits_out, splits_in, group=group)
    # (world, rows, k) -> (rows, world, k): each row's lists point-major
    li = recv_i.view(world, mine, k).transpose(0, 1).contiguous()
    ld = recv_d.view(world, mine, k).transpose(0, 1).contiguous()
    mi, md = merge(li, ld, k)
    if not gather:
        return mi, md, bounds
    m = max(counts)
    pad_i = torch.full((m, k), -1, dtype=mi.dtype, device=mi.device)
    pad_d = torch.full((m, k), float("inf"), dtype=md.dtype, device=md.device)
    pad_i[:mine] = mi
    pad_d[:mine] = md
    all_i = [torch.empty_like(pad_i) for _ in range(world)]
    all_d = [torch.empty_like(pad_d) for _ in range(world)]
    dist_.all_gather(all_i, pad_i, group=group)
    dist_.all_gather(all_d, pad_d, group=group)
    out_i = torch.cat([all_i[r][:counts[r]] for r in range(world)])
    out_d = torch.cat([all_d[r][:counts[r]] for r in range(world)])
    return out_i, out_d, bounds


def build_graph_sharded(data, ntrees: int, nn: int, seed: int, *, group=None,
                        gather: bool = True, **kw):
    """k-NN graph of `data` (a CUDA tensor on this rank's GPU, the same rows on
    every rank) from `ntrees` trees dealt out over the ranks of `group`.
    `kw` are build_graph's options (mode, leaf_size, precision, ...).
    Returns (idx, dist, bounds) as exchange_merge does."""
    torch = _torch()
    import torch.distributed as dist_

    if not _is_cuda_tensor(data):
        raise ValueError("build_graph_sharded takes the rows as a CUDA tensor")
    world = dist_.get_world_size(group)
    rank = dist_.get_rank(group)
    share = tree_share(ntrees, world, rank)
    n = int(data.shape[0])
    if share > 0:
        idx, dist, _ = build_graph(data, share, nn, rank_seed(seed, rank), **kw)
    else:
        idx = torch.full((n, nn), -1, dtype=torch.int32, device=data.device)
        dist = torch.full((n, nn), float("inf"), dtype=torch.float32, device=data.device)
    return exchange_merge(idx, dist, nn, group=group, merge=device_merge, gather=gather)

