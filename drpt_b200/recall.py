"""Recall@k of a k-NN graph against exact neighbours computed in FP64 on the
GPU for a seeded sample of query points (self excluded, ties by index)."""
from __future__ import annotations

import numpy as np


def exact_knn_fp64(X, queries: np.ndarray, k: int, device: int = 0, chunk: int = 512):
    """Exact k nearest neighbours (indices, distances) of X[queries] in X.
    Candidates come from an FP64 norm expansion; the final order uses FP64
    distances recomputed from differences."""
    import torch
    dev = torch.device("cuda", device)
    Xd = X if isinstance(X, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(X))
    Xd = Xd.to(dev).to(torch.float64)
    sq = (Xd * Xd).sum(1)
    out_i = np.empty((len(queries), k), np.int64)
    out_d = np.empty((len(queries), k), np.float64)
    extra = 16
    for s in range(0, len(queries), chunk):
        q = torch.as_tensor(np.asarray(queries[s:s + chunk]), device=dev, dtype=torch.long)
        Q = Xd[q]
        d2 = sq[q][:, None] + sq[None, :] - 2.0 * (Q @ Xd.T)
        d2[torch.arange(len(q), device=dev), q] = float("inf")
        cand = torch.topk(d2, k + extra, dim=1, largest=False).indices  # (b, k+extra)
        diff = Xd[cand] - Q[:, None, :]
        exact = torch.sqrt((diff * diff).sum(-1))
        exact[cand == q[:, None]] = float("inf")
        # order by (distance, index)
        key_idx = torch.argsort(cand, dim=1, stable=True)
        cand_s = torch.gather(cand, 1, key_idx)
        exact_s = torch.gather(exact, 1, key_idx)
        o = torch.argsort(exact_s, dim=1, stable=True)[:, :k]
        out_i[s:s + len(q)] = torch.gather(cand_s, 1, o).cpu().numpy()
        out_d[s:s + len(q)] = torch.gather(exact_s, 1, o).cpu().numpy()
    return out_i, out_d


def recall_at_k(found_idx: np.ndarray, true_idx: np.ndarray) -> float:
    """Fraction of the true k neighbours found among the first k returned."""
    k = true_idx.shape[1]
    f = np.asarray(found_idx)[:, :k]
    hits = sum(len(np.intersect1d(a, b)) for a, b in zip(f, true_idx))
    return hits / true_idx.size


def sample_queries(n: int, count: int = 1000, seed: int = 0) -> np.ndarray:
    return np.sort(np.random.default_rng(seed).choice(n, size=min(count, n), replace=False))
