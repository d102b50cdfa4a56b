"""Python front end of libdrpt_gpu.so.

* ``build_graph`` -- one call for the whole path (drpt_build_graph).
* ``MDRPT`` -- the reference's orchestrator interface (cpp/src/drpt/algo/
  mdrpt.hpp:102-110): construct, ``grow_trees`` (projection, global trees,
  local split) and ``gather_nns`` (leaf brute force and cross-tree merge),
  driven through the kernel-level C entry points.  Errors the reference
  raises as std::out_of_range arrive here as DrptError with status
  DRPT_ERR_DEPTH_OUT_OF_RANGE or DRPT_ERR_EMPTY_LEAF.

PyTorch only supplies device memory and streams.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _lib
from ._lib import DrptError, Stats, check

__all__ = ["build_graph", "build_graph_batched", "build_graph_stream", "build_index", "Index",
           "MDRPT", "DrptError", "edge_list_lines", "global_depth"]


def _torch():
    import torch
    return torch


def _is_cuda_tensor(x) -> bool:
    try:
        torch = _torch()
    except ImportError:
        return False
    return isinstance(x, torch.Tensor) and x.is_cuda


def _dtype_code(x) -> int:
    if _is_cuda_tensor(x):
        torch = _torch()
        if x.dtype == torch.uint8:
            return _lib.DTYPE_U8
        if x.dtype == torch.float32:
            return _lib.DTYPE_F32
    else:
        if x.dtype == np.uint8:
            return _lib.DTYPE_U8
        if x.dtype == np.float32:
            return _lib.DTYPE_F32
    raise TypeError(f"data must be uint8 or float32, got {x.dtype}")


def global_depth(n: int, tree_depth_ratio: float = 0.6, tree_depth: int = 0) -> tuple[int, int]:
    """(tree_depth, global depth) as main.cpp:141-145 and mdrpt.cpp:52 derive them."""
    td = tree_depth if tree_depth > 0 else int(math.log2(n) - 2)
    return td, int(td * tree_depth_ratio)


def build_graph(data, ntrees: int, nn: int, seed: int, *, mode: str = "exact",
                tree_depth_ratio: float = 0.6, local_tree_offset: int = 2, tree_depth: int = 0,
                density: float = 0.0, local_seeds=None, device: int = 0, stream=None,
                out=None, leaf_size: int = 0, precision: str = "bf16", learned_trees: int = 0,
                learn_sample: int = 0, learn_iters: int = 0, locality: bool = False,
                list_width: int = 0, projection: str = "gaussian", _index_out=None):
    """k-NN graph of `data` (n x d, uint8 or float32; a NumPy array in host
    memory or a CUDA tensor).  Returns (idx, dist, stats): idx int32 and dist
    float32 of shape (n, nn), each point's nn nearest distinct neighbours other
    than itself over all trees, ordered by (distance, index), -1/+inf padded;
    device tensors when `data` is one.  `out` = (idx, dist) preallocated
    outputs of the same kind as `data`.  `precision` ("bf16" or "fp8") selects
    the operand type of the mixed form's tensor-core leaf tiles; the last
    `learned_trees` of the `ntrees` trees split on learned MLP values trained
    on a sample of `learn_sample` points (0 = 8,192) with `learn_iters` Adam
    steps per level (0 = 10).  `locality` (exact and fast modes) runs the
    reference's locality relabelling of the global leaves; at one rank the
    graph is the same either way.  `list_width` (mixed mode: 16 or 32, at
    least nn; 0 = 16 for nn <= 10, else 32) is how many candidates per point
    and tree the mixed form keeps for its final FP32 re-rank.  `projection`
    ("gaussian" or "sign"; mixed and fp32_gram modes, uint8 rows with d a
    multiple of 16): "sign" projects with the sign of the reference's sparse
    Gaussian matrix as an exact integer product on the tensor cores."""
    on_dev = _is_cuda_tensor(data)
    if not on_dev:
        data = np.ascontiguousarray(data)
    else:
        data = data.contiguous()
    n, d = int(data.shape[0]), int(data.shape[1])
    desc = _lib.BuildDesc()
    desc.n, desc.d, desc.dtype = n, d, _dtype_code(data)
    desc.ntrees, desc.nn = ntrees, nn
    desc.tree_depth_ratio, desc.local_tree_offset, desc.tree_depth = tree_depth_ratio, \
        local_tree_offset, tree_depth
    desc.density, desc.seed = density, seed & 0xFFFFFFFF
    seeds_arr = None
    if local_seeds is not None:
        seeds_arr = (ctypes.c_uint32 * ntrees)(*[int(s) & 0xFFFFFFFF for s in local_seeds])
        desc.local_seeds = seeds_arr
    desc.mode = {"exact": _lib.MODE_EXACT, "fast": _lib.MODE_FAST, "mixed": _lib.MODE_MIXED,
                 "fp32_leaf": _lib.MODE_FP32_LEAF, "fp32_gram": _lib.MODE_FP32_GRAM}[mode]
    desc.leaf_size = leaf_size
    desc.precision = {"bf16": _lib.PRECISION_BF16, "fp8": _lib.PRECISION_FP8_E4M3}[precision]
    desc.learned_trees, desc.learn_sample = learned_trees, learn_sample
    desc.learn_iters = learn_iters
    desc.locality = 1 if locality else 0
    desc.list_width = list_width
    desc.projection = {"gaussian": _lib.PROJECTION_GAUSSIAN, "sign": _lib.PROJECTION_SIGN}[projection]
    desc.data_on_device = 1 if on_dev else 0
    desc.out_on_device = desc.data_on_device
    if on_dev:
        torch = _torch()
        if stream is None:
            stream = torch.cuda.current_stream(data.device).cuda_stream
        device = data.device.index if data.device.index is not None else 0
        if out is None:
            idx = torch.empty((n, nn), dtype=torch.int32, device=data.device)
            dist = torch.empty((n, nn), dtype=torch.float32, device=data.device)
        else:
            idx, dist = out
        ptr_data, ptr_idx, ptr_dist = data.data_ptr(), idx.data_ptr(), dist.data_ptr()
    else:
        if out is None:
            idx = np.empty((n, nn), np.int32)
            dist = np.empty((n, nn), np.float32)
        else:
            idx, dist = out
        ptr_data, ptr_idx, ptr_dist = data.ctypes.data, idx.ctypes.data, dist.ctypes.data
    desc.stream = stream or 0
    ctx = _lib.context(device)
    stats = Stats()
    if _index_out is not None:
        h = ctypes.c_void_p()
        check(_lib.load().drpt_index_build(ctx.handle, ctypes.byref(desc), ptr_data, ptr_idx,
                                           ptr_dist, ctypes.byref(stats), ctypes.byref(h)))
        _index_out.append(Index(h, device, desc.dtype, d, data))
    else:
        check(_lib.load().drpt_build_graph(ctx.handle, ctypes.byref(desc), ptr_data, ptr_idx,
                                           ptr_dist, ctypes.byref(stats)))
    return idx, dist, stats


def build_graph_stream(datasets, ntrees: int, nn: int, seed: int, *, leaf_size: int = 0,
                       precision: str = "bf16", list_width: int = 0, density: float = 0.0,
                       outs=None, stream=None, device: int = 0):
    """Mixed-form graphs of many same-shape host datasets, pipelined
    (drpt_build_graph_stream): dataset j's copy to the device and the copy of
    dataset j - 1's lists back run on their own streams while graph j is
    built.  `datasets`: NumPy arrays of one shape and dtype (pinned memory
    lets the copies overlap); `outs`: optional list of (idx, dist) host arrays.
    Returns (list of (idx, dist), stats); each graph equals build_graph's of
    the same dataset."""
    datasets = [np.ascontiguousarray(x) for x in datasets]
    if not datasets:
        raise ValueError("no datasets")
    n, d = int(datasets[0].shape[0]), int(datasets[0].shape[1])
    code = _dtype_code(datasets[0])
    for x in datasets:
        if x.shape != datasets[0].shape or _dtype_code(x) != code:
            raise ValueError("every dataset must have the same shape and dtype")
    if outs is None:
        outs = [(np.empty((n, nn), np.int32), np.empty((n, nn), np.float32)) for _ in datasets]
    desc = _lib.BuildDesc()
    desc.n, desc.d, desc.dtype = n, d, code
    desc.ntrees, desc.nn = ntrees, nn
    desc.tree_depth_ratio, desc.local_tree_offset, desc.tree_depth = 0.6, 2, 0
    desc.density, desc.seed = density, seed & 0xFFFFFFFF
    desc.mode = _lib.MODE_MIXED
    desc.leaf_size = leaf_size
    desc.precision = {"bf16": _lib.PRECISION_BF16, "fp8": _lib.PRECISION_FP8_E4M3}[precision]
    desc.list_width = list_width
    desc.data_on_device = desc.out_on_device = 0
    desc.stream = stream or 0
    k = len(datasets)
    data_p = (ctypes.c_void_p * k)(*[x.ctypes.data for x in datasets])
    idx_p = (ctypes.c_void_p * k)(*[o[0].ctypes.data for o in outs])
    dist_p = (ctypes.c_void_p * k)(*[o[1].ctypes.data for o in outs])
    stats = Stats()
    ctx = _lib.context(device)
    check(_lib.load().drpt_build_graph_stream(ctx.handle, ctypes.byref(desc), k, data_p, idx_p,
                                              dist_p, ctypes.byref(stats)))
    return outs, stats


class Index:
    """Trees of a mixed-form build kept for out-of-sample queries
    (drpt_index_build / drpt_index_query).  Holds its own device copies of
    the rows, leaves, node medians and split functions."""

    def __init__(self, handle, device: int, dtype: int, d: int, like):
        self.handle, self.device, self.dtype, self.d = handle, device, dtype, d
        self._cuda = _is_cuda_tensor(like)
        self._lib = _lib.load()

    def query(self, queries, k: int, stream=None):
        """The k (<= 32) nearest indexed points of every query row among the
        members of its leaves, by exact FP32 distance: (idx, dist) of shape
        (nq, k), device tensors for a CUDA tensor argument, NumPy otherwise."""
        on_dev = _is_cuda_tensor(queries)
        q = queries.contiguous() if on_dev else np.ascontiguousarray(queries)
        if _dtype_code(q) != self.dtype or q.shape[1] != self.d:
            raise DrptError(1, "queries must have the index's dtype and dimension")
        nq = int(q.shape[0])
        if on_dev:
            torch = _torch()
            idx = torch.empty((nq, k), dtype=torch.int32, device=q.device)
            dist = torch.empty((nq, k), dtype=torch.float32, device=q.device)
            if stream is None:
                stream = torch.cuda.current_stream(q.device).cuda_stream
            ptrs = (q.data_ptr(), idx.data_ptr(), dist.data_ptr())
        else:
            idx = np.empty((nq, k), np.int32)
            dist = np.empty((nq, k), np.float32)
            ptrs = (q.ctypes.data, idx.ctypes.data, dist.ctypes.data)
        check(self._lib.drpt_index_query(self.handle, ptrs[0], nq, k, 1 if on_dev else 0,
                                         ptrs[1], ptrs[2], stream or 0))
        return idx, dist

    def close(self) -> None:
        if self.handle:
            self._lib.drpt_index_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def build_index(data, ntrees: int, nn: int, seed: int, **kw):
    """build_graph in the mixed form that also returns an Index for
    out-of-sample queries: (index, idx, dist, stats)."""
    kw.setdefault("mode", "mixed")
    box = []
    idx, dist, stats = build_graph(data, ntrees, nn, seed, _index_out=box, **kw)
    return box[0], idx, dist, stats


def build_graph_batched(data, offsets, ntrees: int, nn: int, seed: int, *, mode: str = "mixed",
                        leaf_size: int = 0, precision: str = "bf16", density: float = 0.0,
                        use_graph: bool = False, stream=None, out=None, list_width: int = 0):
    """k-NN graphs of many independent datasets in one call
    (drpt_build_graph_batched).  `data` holds the datasets row after row (a
    NumPy array or a CUDA tensor, uint8 or float32); dataset s is rows
    offsets[s]:offsets[s+1].  Returns (idx, dist, stats) with idx relative to
    each dataset's first row; each dataset's rows equal build_graph on that
    dataset alone.  `use_graph` captures the device work in a CUDA graph and
    replays it on later calls with the same offsets, parameters and tensors
    (CUDA tensors only).  `list_width` as in build_graph."""
    offs = np.ascontiguousarray(np.asarray(offsets, dtype=np.int64))
    on_dev = _is_cuda_tensor(data)
    data = data.contiguous() if on_dev else np.ascontiguousarray(data)
    n, d = int(data.shape[0]), int(data.shape[1])
    if offs[-1] != n:
        raise DrptError(1, f"offsets end at {offs[-1]}, data has {n} rows")
    desc = _lib.BatchDesc()
    desc.nsets, desc.d, desc.dtype = len(offs) - 1, d, _dtype_code(data)
    desc.ntrees, desc.nn = ntrees, nn
    desc.mode = {"mixed": _lib.MODE_MIXED, "fp32_leaf": _lib.MODE_FP32_LEAF}[mode]
    desc.precision = {"bf16": _lib.PRECISION_BF16, "fp8": _lib.PRECISION_FP8_E4M3}[precision]
    desc.list_width = list_width
    desc.leaf_size, desc.seed, desc.density = leaf_size, seed & 0xFFFFFFFF, density
    desc.use_graph = 1 if use_graph else 0
    desc.data_on_device = desc.out_on_device = 1 if on_dev else 0
    if on_dev:
        torch = _torch()
        if stream is None:
            stream = torch.cuda.current_stream(data.device).cuda_stream
        device = data.device.index if data.device.index is not None else 0
        if out is None:
            idx = torch.empty((n, nn), dtype=torch.int32, device=data.device)
            dist = torch.empty((n, nn), dtype=torch.float32, device=data.device)
        else:
            idx, dist = out
        ptrs = (data.data_ptr(), idx.data_ptr(), dist.data_ptr())
    else:
        device = 0
        if out is None:
            idx = np.empty((n, nn), np.int32)
            dist = np.empty((n, nn), np.float32)
        else:
            idx, dist = out
        ptrs = (data.ctypes.data, idx.ctypes.data, dist.ctypes.data)
    desc.stream = stream or 0
    ctx = _lib.context(device)
    stats = Stats()
    check(_lib.load().drpt_build_graph_batched(ctx.handle, ctypes.byref(desc), offs.ctypes.data,
                                               ptrs[0], ptrs[1], ptrs[2], ctypes.byref(stats)))
    return idx, dist, stats


def edge_list_lines(idx: np.ndarray, nn: int) -> list[str]:
    """The reference's edge-list text (file_writer.cpp:95-149): for every
    source in ascending order, its first `nn` neighbours as 1-based
    "src dst" lines.  The reference CLI passes nn-1 (main.cpp:228)."""
    lines = []
    for p in range(idx.shape[0]):
        for q in idx[p, :nn]:
            if q < 0:
                break
            lines.append(f"{p + 1} {int(q) + 1}")
    return lines


class MDRPT:
    """The reference's MDRPT interface on one GPU (rank 0 of 1).

    Arguments keep the reference's names and meaning (mdrpt.hpp:102-105);
    `seed` and `local_seeds` replace the std::random_device draws of
    receive_random_seeds (mdrpt.cpp:402-416).  Data live on `device`."""

    def __init__(self, ntrees: int, tree_depth: int, tree_depth_ratio: float,
                 local_tree_offset: int, total_data_set_size: int, local_data_set_size: int,
                 dimension: int, rank: int = 0, world_size: int = 1, input_path: str = "",
                 output_path: str = "", *, seed: int = 0, local_seeds=None, exact: bool = True,
                 device: int = 0):
        if world_size != 1 or rank != 0:
            raise DrptError(1, "one GPU process: world_size must be 1")
        self.ntrees, self.tree_depth, self.tree_depth_ratio = ntrees, tree_depth, tree_depth_ratio
        self.local_tree_offset = local_tree_offset
        self.n, self.d = int(local_data_set_size), int(dimension)
        if total_data_set_size != local_data_set_size:
            raise DrptError(1, "one rank holds every point")
        self.seed, self.local_seeds = seed & 0xFFFFFFFF, local_seeds
        self.exact, self.device = exact, device
        self.input_path, self.output_path = input_path, output_path
        self._ctx = _lib.context(device)
        self._L = _lib.load()

    def _stream(self):
        return _torch().cuda.current_stream(self.device).cuda_stream

    def grow_trees(self, original_data, density: float, use_locality_optimization: bool, nn: int):
        """Projection, global trees and positional local split
        (mdrpt.cpp:46-121).  With `use_locality_optimization` the global
        leaves are put in the reference's locality slot order
        (drpt_global.cpp:572-732) before the local split; at one rank that
        only renumbers leaves, the graph is the same."""
        torch = _torch()
        dev = torch.device("cuda", self.device)
        X = original_data if _is_cuda_tensor(original_data) else \
            torch.from_numpy(np.ascontiguousarray(original_data)).to(dev)
        X = X.contiguous()
        self.X, self.dtype_code = X, _dtype_code(X)
        n, d, T = self.n, self.d, self.ntrees
        gd = int(self.tree_depth * self.tree_depth_ratio)
        if gd <= 0 or gd > math.log2(n):
            raise DrptError(2, f"global depth {gd} outside [1, log2({n})]")
        self.gd = gd
        density = density if density else 1.0 / math.sqrt(d)
        L = gd * T
        B = np.empty((d, L), np.float32)
        check(self._L.drpt_host_projection(self.seed, d, L, ctypes.c_float(density),
                                           B.ctypes.data))
        self.B = B
        s = self._stream()
        cols = np.array([t * gd + lv for t in range(T) for lv in range(gd - 1)], np.int32)
        P = torch.empty((max(len(cols), 1), n), dtype=torch.float32, device=dev)
        if len(cols):
            check(self._L.drpt_project(self._ctx.handle, X.data_ptr(), n, d, self.dtype_code,
                                       B.ctypes.data, L, cols.ctypes.data, len(cols),
                                       P.data_ptr(), s))
        nleaf = 1 << (gd - 1)
        order = torch.empty((T, n), dtype=torch.int32, device=dev)
        offs = torch.empty((T, nleaf + 1), dtype=torch.int32, device=dev)
        med = torch.empty((T, max(nleaf - 1, 1)), dtype=torch.float32, device=dev)
        check(self._L.drpt_global_trees(self._ctx.handle, P.data_ptr(), n, T, gd,
                                        1 if self.exact else 0, order.data_ptr(), offs.data_ptr(),
                                        med.data_ptr(), s))
        if use_locality_optimization:
            ho = np.ascontiguousarray(order.cpu().numpy())
            hf = np.ascontiguousarray(offs.cpu().numpy())
            slots = np.empty((nleaf, T), np.int32)
            so, sf = np.empty_like(ho), np.empty_like(hf)
            check(self._L.drpt_locality_slots(ho.ctypes.data, hf.ctypes.data, n, T, nleaf,
                                              slots.ctypes.data, so.ctypes.data, sf.ctypes.data))
            self.locality_slots = slots
            order = torch.from_numpy(so).to(dev)
            offs = torch.from_numpy(sf).to(dev)
        self.P, self.global_order, self.global_offsets, self.medians = P, order, offs, med
        sizes = (offs[:, 1:] - offs[:, :-1]).cpu().numpy()
        nonempty = sizes[sizes > 0]
        min_leaf = int(nonempty.min())
        ld = int(math.log2(min_leaf) - (math.log2(nn) + self.local_tree_offset))
        if ld <= 0:
            raise DrptError(2, f"local tree depth {ld} <= 0")
        if (sizes == 0).any():
            raise DrptError(3, "a global leaf is empty")
        self.ld = ld
        n_final = nleaf << ld
        forder = torch.empty((T, n), dtype=torch.int32, device=dev)
        foffs = torch.empty((T, n_final + 1), dtype=torch.int32, device=dev)
        check(self._L.drpt_local_leaves(self._ctx.handle, order.data_ptr(), offs.data_ptr(), n, T,
                                        gd, ld, forder.data_ptr(), foffs.data_ptr(), s))
        self.final_order, self.final_offsets, self.n_final = forder, foffs, n_final

    def gather_nns(self, nn: int):
        """Leaf brute force and merge (mdrpt.cpp:273-291).  Returns device
        tensors (idx, dist) of shape (n, nn)."""
        torch = _torch()
        dev = torch.device("cuda", self.device)
        n, T = self.n, self.ntrees
        s = self._stream()
        cidx = torch.empty((n, T, nn), dtype=torch.int32, device=dev)
        cdist = torch.empty((n, T, nn), dtype=torch.float32, device=dev)
        check(self._L.drpt_leaf_knn(self._ctx.handle, self.X.data_ptr(), self.dtype_code, n, self.d,
                                    T, self.final_order.data_ptr(), self.final_offsets.data_ptr(),
                                    self.n_final, nn, cidx.data_ptr(), cdist.data_ptr(), s))
        idx = torch.empty((n, nn), dtype=torch.int32, device=dev)
        dist = torch.empty((n, nn), dtype=torch.float32, device=dev)
        check(self._L.drpt_merge_candidates(self._ctx.handle, cidx.data_ptr(), cdist.data_ptr(), n,
                                            T, nn, idx.data_ptr(), dist.data_ptr(), s))
        self.cand_idx, self.cand_dist = cidx, cdist
        return idx, dist
