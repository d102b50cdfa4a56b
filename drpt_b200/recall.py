"""Recall@k of a k-NN graph against exact neighbours computed in FP64 on the
GPU for a seeded sample of query points (self excluded, ties by index)."""
from __future__ import annotations

import numpy as np


def exact_knn_fp64(X, queries: np.ndarray, k: int, device=0, chunk: int = 512):
    """Exact k nearest neighbours (indices, distances) of X[queries] in X,
    self excluded, ordered by (distance, index), distances in FP64 from
    differences.  `device`: a CUDA device number, or "cpu".

    Candidates come from an FP64 norm expansion (k + 16 smallest); a row is
    settled from them only when the 16 extra candidates separate the k-th
    from every point left out by more than twice the expansion's rounding
    bound.  Otherwise (exact or near ties at the boundary, as integer data
    has) the row is recomputed from differences over all points and sorted
    in full, so the result is the brute-force one in every case."""
    import torch
    dev = torch.device("cpu") if device == "cpu" else torch.device("cuda", device)
    Xd = X if isinstance(X, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(X))
    Xd = Xd.to(dev).to(torch.float64)
    n = Xd.shape[0]
    sq = (Xd * Xd).sum(1)
    sq_max = float(sq.max()) if n else 0.0
    out_i = np.empty((len(queries), k), np.int64)
    out_d = np.empty((len(queries), k), np.float64)
    extra = min(16, max(n - 1 - k, 0))
    ar = torch.arange(n, device=dev)
    for s in range(0, len(queries), chunk):
        q = torch.as_tensor(np.asarray(queries[s:s + chunk]), device=dev, dtype=torch.long)
        Q = Xd[q]
        d2 = sq[q][:, None] + sq[None, :] - 2.0 * (Q @ Xd.T)
        d2[torch.arange(len(q), device=dev), q] = float("inf")
        top = torch.topk(d2, k + extra, dim=1, largest=False)
        cand = top.indices  # (b, k+extra), ascending expanded d2
        # rounding bound of the expansion (a few ulp of |q|^2 + |x|^2, taken generously)
        err = 1e-12 * (sq[q] + sq_max + 1.0)
        settled = (top.values[:, -1] - top.values[:, k - 1]) > 2.0 * err if extra else             torch.ones(len(q), dtype=torch.bool, device=dev)
        diff = Xd[cand] - Q[:, None, :]
        exact = torch.sqrt((diff * diff).sum(-1))
        exact[cand == q[:, None]] = float("inf")
        # order by (distance, index)
        key_idx = torch.argsort(cand, dim=1, stable=True)
        cand_s = torch.gather(cand, 1, key_idx)
        exact_s = torch.gather(exact, 1, key_idx)
        o = torch.argsort(exact_s, dim=1, stable=True)[:, :k]
        bi = torch.gather(cand_s, 1, o)
        bd = torch.gather(exact_s, 1, o)
        for r in torch.nonzero(~settled).flatten().tolist():
            df = Xd - Q[r]
            full = torch.sqrt((df * df).sum(1))
            full[q[r]] = float("inf")
            oo = torch.argsort(full, stable=True)[:k]  # ties stay in index order
            bi[r] = ar[oo]
            bd[r] = full[oo]
        out_i[s:s + len(q)] = bi.cpu().numpy()
        out_d[s:s + len(q)] = bd.cpu().numpy()
    return out_i, out_d


def recall_at_k(found_idx: np.ndarray, true_idx: np.ndarray) -> float:
    """Fraction of the true k neighbours found among the first k returned."""
    k = true_idx.shape[1]
    f = np.asarray(found_idx)[:, :k]
    hits = sum(len(np.intersect1d(a, b)) for a, b in zip(f, true_idx))
    return hits / true_idx.size


def sample_queries(n: int, count: int = 1000, seed: int = 0) -> np.ndarray:
    return np.sort(np.random.default_rng(seed).choice(n, size=min(count, n), replace=False))
