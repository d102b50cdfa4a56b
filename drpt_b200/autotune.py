"""Autotuner of the mixed form's leaf phase.

Two settings decide how much work the tensor-core leaf kernel and the
re-rank do, and how much recall they keep:

* the target global-leaf size, which sets how many 128 x 64 Gram tiles each
  leaf has (the work grows with the leaf size, so does recall);
* the list width, 16 or 32 candidates per point and tree: the top-k width of
  the leaf kernel's epilogue (16 keys fit three CTAs per SM, 32 keys two)
  and the number of rows the FP32 re-rank reads per point.

The tuner builds the caller's own data with each candidate setting, times the
builds with CUDA events (after one untimed build; batched builds replay their
CUDA graph as production calls do), measures recall@10 against exact FP64
neighbours of a seeded query sample, and keeps the fastest setting that
reaches the target recall (the most accurate one if none does).  A result can
be cached in a JSON file under a key made of the problem's shape and
parameters, so that repeated runs of the same problem skip the search.
"""
from __future__ import annotations

import hashlib
import json
import os
import time

import numpy as np

from . import recall as _recall
from .graph import _is_cuda_tensor, _torch, build_graph, build_graph_batched


def choose(trials: list[dict], target_recall: float) -> dict:
    """The fastest trial whose recall reaches `target_recall`, else the trial
    with the best recall (ties: the faster)."""
    ok = [t for t in trials if t["recall"] >= target_recall]
    if ok:
        return min(ok, key=lambda t: (t["ms"], -t["recall"]))
    return max(trials, key=lambda t: (t["recall"], -t["ms"]))


def _widths(nn: int, widths) -> list[int]:
    ws = [w for w in (widths or (16, 32)) if w in (16, 32) and w >= nn]
    if not ws:
        raise ValueError(f"no list width in {widths} holds nn = {nn} neighbours")
    return ws


def _load_cache(path, key):
    if path and os.path.exists(path):
        try:
            return json.load(open(path)).get(key)
        except (OSError, ValueError):
            return None
    return None


def _store_cache(path, key, value):
    if not path:
        return
    try:
        table = json.load(open(path)) if os.path.exists(path) else {}
    except (OSError, ValueError):
        table = {}
    table[key] = value
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def _timed(torch, fn, reps: int) -> float:
    fn()  # untimed: first-call set-up (workspace, graph capture)
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(s)
    for _ in range(reps):
        fn()
    e1.record(s)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def tune_batched(data, offsets, ntrees: int, nn: int, seed: int, *, target_recall: float = 0.90,
                 leaf_sizes=(256, 512, 1024), widths=None, precision: str = "bf16",
                 reps: int = 2, sample_sets: int = 8, queries_per_set: int = 50,
                 cache_path: str | None = None) -> dict:
    """Leaf size and list width for build_graph_batched(data, offsets, ntrees,
    nn, seed, mode="mixed", ...) on a CUDA tensor `data`.  Returns a dict with
    `leaf_size`, `list_width`, `ms`, `recall`, `trials` and `tune_s`."""
    torch = _torch()
    if not _is_cuda_tensor(data):
        raise ValueError("tune_batched takes the rows as a CUDA tensor")
    offs = np.ascontiguousarray(np.asarray(offsets, dtype=np.int64))
    n, d = int(data.shape[0]), int(data.shape[1])
    nsets = len(offs) - 1
    sig = hashlib.sha1(offs.tobytes()).hexdigest()[:16]
    key = (f"batched:{nsets}:{n}:{d}:{data.dtype}:{ntrees}:{nn}:{precision}:{target_recall}:"
           f"{tuple(leaf_sizes)}:{tuple(_widths(nn, widths))}:{sig}")
    hit = _load_cache(cache_path, key)
    if hit is not None:
        return dict(hit, cached=True)
    t0 = time.perf_counter()
    k = min(10, nn)
    picks = np.unique(np.linspace(0, nsets - 1, min(sample_sets, nsets)).round().astype(int))
    truth = []
    for s in picks:
        x = data[offs[s]:offs[s + 1]]
        q = _recall.sample_queries(len(x), queries_per_set, seed=int(s))
        ti, _ = _recall.exact_knn_fp64(x, q, k, device=data.device.index or 0)
        truth.append((int(s), q, ti))
    idx = torch.empty((n, nn), dtype=torch.int32, device=data.device)
    dist = torch.empty((n, nn), dtype=torch.float32, device=data.device)
    trials = []
    for leaf in leaf_sizes:
        for w in _widths(nn, widths):
            def run(leaf=leaf, w=w):
                return build_graph_batched(data, offs, ntrees, nn, seed, mode="mixed",
                                           leaf_size=leaf, precision=precision, use_graph=True,
                                           out=(idx, dist), list_width=w)
            ms = _timed(torch, run, reps)
            hits = 0
            for s, q, ti in truth:
                got = idx[offs[s]:offs[s + 1]].cpu().numpy()[q][:, :k]
                hits += _recall.recall_at_k(got, ti) * ti.size
            rec = hits / sum(ti.size for _, _, ti in truth)
            trials.append({"leaf_size": int(leaf), "list_width": int(w), "ms": float(ms),
                           "recall": float(rec)})
    best = choose(trials, target_recall)
    out = {"leaf_size": best["leaf_size"], "list_width": best["list_width"], "ms": best["ms"],
           "recall": best["recall"], "target_recall": target_recall, "trials": trials,
           "tune_s": time.perf_counter() - t0}
    _store_cache(cache_path, key, out)
    return dict(out, cached=False)


def tune_graph(data, ntrees: int, nn: int, seed: int, *, target_recall: float = 0.90,
               leaf_sizes=(512, 1024, 2048), widths=None, precision: str = "bf16",
               reps: int = 2, queries: int = 500, cache_path: str | None = None) -> dict:
    """Leaf size and list width for build_graph(data, ntrees, nn, seed,
    mode="mixed", ...) on a CUDA tensor `data`; returns what tune_batched
    returns."""
    torch = _torch()
    if not _is_cuda_tensor(data):
        raise ValueError("tune_graph takes the rows as a CUDA tensor")
    n, d = int(data.shape[0]), int(data.shape[1])
    key = (f"single:{n}:{d}:{data.dtype}:{ntrees}:{nn}:{precision}:{target_recall}:"
           f"{tuple(leaf_sizes)}:{tuple(_widths(nn, widths))}")
    hit = _load_cache(cache_path, key)
    if hit is not None:
        return dict(hit, cached=True)
    t0 = time.perf_counter()
    k = min(10, nn)
    q = _recall.sample_queries(n, queries, seed=0)
    ti, _ = _recall.exact_knn_fp64(data, q, k, device=data.device.index or 0)
    idx = torch.empty((n, nn), dtype=torch.int32, device=data.device)
    dist = torch.empty((n, nn), dtype=torch.float32, device=data.device)
    trials = []
    for leaf in leaf_sizes:
        for w in _widths(nn, widths):
            def run(leaf=leaf, w=w):
                return build_graph(data, ntrees, nn, seed, mode="mixed", leaf_size=leaf,
                                   precision=precision, out=(idx, dist), list_width=w)
            ms = _timed(torch, run, reps)
            rec = _recall.recall_at_k(idx.cpu().numpy()[q][:, :k], ti)
            trials.append({"leaf_size": int(leaf), "list_width": int(w), "ms": float(ms),
                           "recall": float(rec)})
    best = choose(trials, target_recall)
    out = {"leaf_size": best["leaf_size"], "list_width": best["list_width"], "ms": best["ms"],
           "recall": best["recall"], "target_recall": target_recall, "trials": trials,
           "tune_s": time.perf_counter() - t0}
    _store_cache(cache_path, key, out)
    return dict(out, cached=False)
