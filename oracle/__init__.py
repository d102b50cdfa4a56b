"""CPU oracle for the DRPT k-NN-graph path -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this package, and only as a checker.  The product (``drpt_b200`` and
``libdrpt_gpu.so``) never imports, links or calls anything here.

* ``libdrpt_oracle.so`` (drpt_oracle.cpp): a plain restatement of the
  reference algorithm, pinned against the reference itself through the golden
  fixtures in tests/golden/.
* ``_ref/drpt_ref``: the reference sources built unmodified with a one-rank
  MPI stand-in, an ordered cblas and seed injection (``make -C oracle ref``;
  only where the reference tree is present).
* ``exact_knn``: FP64 brute-force k-NN, the recall oracle.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdrpt_oracle.so")
REF_BIN = os.path.join(HERE, "_ref", "drpt_ref")

_lib = None


class Desc(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("d", ctypes.c_int), ("is_u8", ctypes.c_int),
                ("ntrees", ctypes.c_int), ("nn", ctypes.c_int),
                ("tree_depth_ratio", ctypes.c_double), ("local_tree_offset", ctypes.c_int),
                ("density", ctypes.c_double), ("seed", ctypes.c_uint32)]


class Info(ctypes.Structure):
    _fields_ = [("tree_depth", ctypes.c_int), ("global_depth", ctypes.c_int),
                ("local_depth", ctypes.c_int), ("n_global_leaves", ctypes.c_int),
                ("n_final_leaves", ctypes.c_int), ("min_global_leaf", ctypes.c_int64)]


def build_lib(reference_root: str | None = None) -> None:
    """Compile libdrpt_oracle.so with the recipe in oracle/Makefile and, when
    a reference checkout is named (`reference_root`, else the environment's
    DRPT_REFERENCE_ROOT), the reference binary _ref/drpt_ref from its
    sources (and _ref/drpt_ref_openblas, the same on OpenBLAS, for timing)
    and, once libdrpt_gpu.so exists, the reference-side binding's
    test driver _ref/adapter_check.  A named root that is not a directory is an error; with none
    named the reference binary is not built."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    root = reference_root or os.environ.get("DRPT_REFERENCE_ROOT")
    if not root:
        return
    if not os.path.isdir(root):
        raise FileNotFoundError(f"reference checkout {root!r} (DRPT_REFERENCE_ROOT) not found")
    subprocess.run(["make", "-s", "-C", HERE, "ref", "REF_ROOT=" + root], check=True)
    # the same build on OpenBLAS (numpy's bundled copy), for the timed CPU
    # baseline only; skipped where numpy ships no OpenBLAS
    subprocess.run(["make", "-s", "-C", HERE, "ref-openblas", "REF_ROOT=" + root,
                    "PYTHON=" + sys.executable], check=False)
    # the reference-side binding of the library, where the library is built
    if os.path.exists(os.path.join(os.path.dirname(HERE), "drpt_b200", "libdrpt_gpu.so")):
        subprocess.run(["make", "-s", "-C", HERE, "adapter", "REF_ROOT=" + root], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build_lib()
        L = ctypes.CDLL(LIB_PATH)
        f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
        i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
        f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
        L.drpt_oracle_projection_matrix.argtypes = [ctypes.c_uint32, ctypes.c_int, ctypes.c_int,
                                                    ctypes.c_float, f32p]
        L.drpt_oracle_project_f32.argtypes = [f32p, ctypes.c_int64, ctypes.c_int, f32p,
                                              ctypes.c_int, f32p]
        L.drpt_oracle_project_u8.argtypes = [np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS"),
                                             ctypes.c_int64, ctypes.c_int, f32p, ctypes.c_int, f32p]
        L.drpt_oracle_node_median.argtypes = [f32p, ctypes.c_int64, f32p, f32p, f64p]
        L.drpt_oracle_global_tree.argtypes = [f32p, ctypes.c_int64, ctypes.c_int, ctypes.c_int,
                                              i32p, i32p, f32p]
        L.drpt_oracle_global_tree.restype = ctypes.c_int
        L.drpt_oracle_local_depth.argtypes = [ctypes.c_int64, ctypes.c_int, ctypes.c_int]
        L.drpt_oracle_local_depth.restype = ctypes.c_int
        L.drpt_oracle_local_perm.argtypes = [ctypes.c_int64, ctypes.c_int, i32p, i32p]
        L.drpt_oracle_local_perm.restype = ctypes.c_int
        L.drpt_oracle_distance.argtypes = [f32p, f32p, ctypes.c_int]
        L.drpt_oracle_distance.restype = ctypes.c_float
        L.drpt_oracle_build.argtypes = [ctypes.POINTER(Desc), ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.POINTER(Info), ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_void_p, ctypes.c_void_p]
        L.drpt_oracle_build.restype = ctypes.c_int
        _lib = L
    return _lib


def projection_matrix(seed: int, d: int, L: int, density: float) -> np.ndarray:
    B = np.empty((d, L), np.float32)
    lib().drpt_oracle_projection_matrix(seed & 0xFFFFFFFF, d, L, np.float32(density), B)
    return B


def project(X: np.ndarray, B: np.ndarray) -> np.ndarray:
    n, d = X.shape
    L = B.shape[1]
    P = np.empty((n, L), np.float32)
    B = np.ascontiguousarray(B, np.float32)
    if X.dtype == np.uint8:
        lib().drpt_oracle_project_u8(np.ascontiguousarray(X), n, d, B, L, P)
    else:
        lib().drpt_oracle_project_f32(np.ascontiguousarray(X, np.float32), n, d, B, L, P)
    return P


def node_median(vals: np.ndarray):
    vals = np.ascontiguousarray(vals, np.float32)
    out4 = np.empty(4, np.float32)
    bounds = np.empty(16, np.float32)
    counts = np.empty(16, np.float64)
    lib().drpt_oracle_node_median(vals, len(vals), out4, bounds, counts)
    return out4, bounds, counts


def global_tree(P: np.ndarray, T: int, gd: int):
    n = P.shape[0]
    nleaf = 1 << (gd - 1)
    order = np.empty(T * n, np.int32)
    offsets = np.empty(T * (nleaf + 1), np.int32)
    medians = np.empty(T * max(nleaf - 1, 1), np.float32)
    st = lib().drpt_oracle_global_tree(np.ascontiguousarray(P, np.float32), n, T, gd, order,
                                       offsets, medians)
    if st:
        raise RuntimeError(f"oracle global_tree status {st}")
    return order.reshape(T, n), offsets.reshape(T, nleaf + 1), medians


def local_perm(n: int, ld: int):
    perm = np.empty(max(n, 1), np.int32)
    first = np.empty((1 << ld) + 1, np.int32)
    st = lib().drpt_oracle_local_perm(n, ld, perm, first)
    if st:
        raise RuntimeError(f"oracle local_perm status {st}")
    return perm[:n], first


def distance(p: np.ndarray, q: np.ndarray) -> float:
    return float(lib().drpt_oracle_distance(np.ascontiguousarray(p, np.float32),
                                            np.ascontiguousarray(q, np.float32), len(p)))


def build(X: np.ndarray, ntrees: int, nn: int, seed: int, tree_depth_ratio: float = 0.6,
          local_tree_offset: int = 2, density: float = 0.0, local_seeds=None, want_knn=True):
    """Whole path on the CPU.  Returns a dict with info, final_order (T x n),
    final_offsets (T x n_final+1) and, when asked, knn_idx / knn_dist."""
    X = np.ascontiguousarray(X)
    n, d = X.shape
    desc = Desc(n, d, 1 if X.dtype == np.uint8 else 0, ntrees, nn, tree_depth_ratio,
                local_tree_offset, density, seed & 0xFFFFFFFF)
    if X.dtype != np.uint8:
        X = np.ascontiguousarray(X, np.float32)
    info = Info()
    order = np.empty(ntrees * n, np.int32)
    offs = np.empty(ntrees * (n + 1), np.int32)
    kidx = np.empty(n * nn, np.int32) if want_knn else None
    kdist = np.empty(n * nn, np.float32) if want_knn else None
    ls = None
    if local_seeds is not None:
        ls = np.ascontiguousarray(np.asarray(local_seeds, np.uint32))
    st = lib().drpt_oracle_build(ctypes.byref(desc), X.ctypes.data,
                                 ls.ctypes.data if ls is not None else None, ctypes.byref(info),
                                 order.ctypes.data, offs.ctypes.data,
                                 kidx.ctypes.data if want_knn else None,
                                 kdist.ctypes.data if want_knn else None)
    out = {"status": st, "info": info}
    if st == 0:
        nf = info.n_final_leaves
        out["final_order"] = order.reshape(ntrees, n)
        out["final_offsets"] = offs[: ntrees * (nf + 1)].reshape(ntrees, nf + 1)
        if want_knn:
            out["knn_idx"] = kidx.reshape(n, nn)
            out["knn_dist"] = kdist.reshape(n, nn)
    return out


def exact_knn(X: np.ndarray, queries: np.ndarray, k: int, chunk: int = 256):
    """FP64 brute-force k nearest neighbours of the query points (indices into
    X), self excluded; ties ordered by index.  Returns (idx, dist).

    Candidates come from an FP64 norm expansion (k + 8 smallest); a row whose
    8 extra candidates do not separate the k-th from the rest by more than
    twice the expansion's rounding bound (ties or near-ties at the boundary)
    is recomputed from differences over all points."""
    Xd = np.asarray(X, np.float64)
    n = len(Xd)
    sq = np.einsum("ij,ij->i", Xd, Xd)
    sq_max = float(sq.max()) if n else 0.0
    extra = min(8, max(n - 1 - k, 0))
    idx_out = np.empty((len(queries), k), np.int64)
    dist_out = np.empty((len(queries), k), np.float64)
    for s in range(0, len(queries), chunk):
        q = np.asarray(queries[s:s + chunk])
        Q = Xd[q]
        d2 = sq[q][:, None] + sq[None, :] - 2.0 * (Q @ Xd.T)
        d2[np.arange(len(q)), q] = np.inf
        part = np.argpartition(d2, k + extra - 1, axis=1)[:, : k + extra] if extra else \
            np.argsort(d2, axis=1, kind="stable")[:, :k]
        for r in range(len(q)):
            cand = part[r]
            vals = np.sort(d2[r, cand])
            err = 1e-12 * (sq[q[r]] + sq_max + 1.0)
            if extra and not (vals[-1] - vals[k - 1] > 2.0 * err):
                cand = np.arange(n)  # ambiguous boundary: every point, from differences
            diff = Xd[cand] - Q[r]
            exact = np.sqrt(np.einsum("ij,ij->i", diff, diff))
            exact[cand == q[r]] = np.inf
            o = np.lexsort((cand, exact))[:k]
            idx_out[s + r] = cand[o]
            dist_out[s + r] = exact[o]
    return idx_out, dist_out


def recall_at_k(found_idx: np.ndarray, true_idx: np.ndarray) -> float:
    """Fraction of the true k nearest neighbours present among the first k
    returned neighbours (self excluded on both sides)."""
    k = true_idx.shape[1]
    hits = 0
    for f, t in zip(found_idx[:, :k], true_idx):
        hits += len(np.intersect1d(f, t, assume_unique=False))
    return hits / true_idx.size
