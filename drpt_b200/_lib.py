"""ctypes binding of libdrpt_gpu.so (the C ABI declared in include/drpt_gpu.h).

The shared library is built in-tree (``python -m drpt_b200.build``).  If it is
missing, loading fails loudly: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
import threading

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libdrpt_gpu.so")

DRPT_OK = 0
STATUS_NAMES = {
    0: "DRPT_OK", 1: "DRPT_ERR_INVALID_ARG", 2: "DRPT_ERR_DEPTH_OUT_OF_RANGE",
    3: "DRPT_ERR_EMPTY_LEAF", 4: "DRPT_ERR_LOCAL_MATRIX_NONZERO", 5: "DRPT_ERR_OOM",
    6: "DRPT_ERR_CUDA", 7: "DRPT_ERR_TIMEOUT", 8: "DRPT_ERR_UNSUPPORTED",
}
DTYPE_F32, DTYPE_U8 = 0, 1
MODE_EXACT, MODE_FAST, MODE_MIXED, MODE_FP32_LEAF, MODE_FP32_GRAM = 0, 1, 2, 3, 4
PRECISION_BF16, PRECISION_FP8_E4M3 = 0, 1

# Every symbol include/drpt_gpu.h declares.
EXPORTS = [
    "drpt_version", "drpt_last_error", "drpt_ctx_create", "drpt_ctx_destroy", "drpt_build_graph",
    "drpt_host_projection", "drpt_project", "drpt_global_trees", "drpt_local_leaves",
    "drpt_leaf_knn", "drpt_merge_candidates", "drpt_global_trees_noalloc",
    "drpt_build_graph_batched", "drpt_learn_gradient", "drpt_index_build", "drpt_index_query",
    "drpt_index_destroy", "drpt_locality_slots", "drpt_build_graph_stream", "drpt_project_sign",
]
PROJECTION_GAUSSIAN, PROJECTION_SIGN = 0, 1


class DrptError(RuntimeError):
    """A libdrpt_gpu call returned a status other than DRPT_OK."""

    def __init__(self, status: int, message: str):
        self.status = status
        self.status_name = STATUS_NAMES.get(status, str(status))
        super().__init__(f"{self.status_name}: {message}")


class BuildDesc(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int64), ("d", ctypes.c_int32), ("dtype", ctypes.c_int32),
        ("ntrees", ctypes.c_int32), ("nn", ctypes.c_int32), ("tree_depth_ratio", ctypes.c_double),
        ("local_tree_offset", ctypes.c_int32), ("tree_depth", ctypes.c_int32),
        ("density", ctypes.c_double), ("seed", ctypes.c_uint32),
        ("local_seeds", ctypes.POINTER(ctypes.c_uint32)), ("mode", ctypes.c_int32),
        ("data_on_device", ctypes.c_int32), ("out_on_device", ctypes.c_int32),
        ("stream", ctypes.c_void_p), ("leaf_size", ctypes.c_int32), ("precision", ctypes.c_int32),
        ("learned_trees", ctypes.c_int32), ("learn_sample", ctypes.c_int32),
        ("learn_iters", ctypes.c_int32), ("locality", ctypes.c_int32),
        ("list_width", ctypes.c_int32), ("projection", ctypes.c_int32),
    ]


class BatchDesc(ctypes.Structure):
    _fields_ = [
        ("nsets", ctypes.c_int32), ("d", ctypes.c_int32), ("dtype", ctypes.c_int32),
        ("ntrees", ctypes.c_int32), ("nn", ctypes.c_int32), ("mode", ctypes.c_int32),
        ("precision", ctypes.c_int32), ("leaf_size", ctypes.c_int32), ("seed", ctypes.c_uint32),
        ("use_graph", ctypes.c_int32), ("density", ctypes.c_double),
        ("data_on_device", ctypes.c_int32), ("out_on_device", ctypes.c_int32),
        ("stream", ctypes.c_void_p), ("list_width", ctypes.c_int32), ("reserved", ctypes.c_int32),
    ]


class Stats(ctypes.Structure):
    _fields_ = [
        ("tree_depth", ctypes.c_int32), ("global_depth", ctypes.c_int32),
        ("local_depth", ctypes.c_int32), ("n_global_leaves", ctypes.c_int32),
        ("n_final_leaves", ctypes.c_int32), ("max_final_leaf", ctypes.c_int32),
        ("min_global_leaf", ctypes.c_int64), ("sum_leaf_sq", ctypes.c_int64),
        ("kernels_launched", ctypes.c_int32), ("reserved", ctypes.c_int32),
        ("ms_project", ctypes.c_float), ("ms_global", ctypes.c_float), ("ms_local", ctypes.c_float),
        ("ms_leaf_knn", ctypes.c_float), ("ms_merge", ctypes.c_float), ("ms_total", ctypes.c_float),
        ("ms_leaf_mma", ctypes.c_float), ("ms_leaf_stage", ctypes.c_float),
        ("mma_pairs_padded", ctypes.c_int64),
        ("ms_learn", ctypes.c_float), ("learn_loss_start", ctypes.c_float),
        ("learn_loss_end", ctypes.c_float), ("reserved2", ctypes.c_int32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_
                if not name.startswith("reserved")}


_lib = None
_lock = threading.Lock()


def load(path: str = LIB_PATH):
    """Load the shared library (and declare its signatures) once."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(path):
            raise RuntimeError(
                f"{path} is missing: build it with `python -m drpt_b200.build` (the k-NN-graph path "
                "has no CPU fallback)")
        L = ctypes.CDLL(path)
        vp, i32, i64, u32 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_uint32
        L.drpt_version.restype = ctypes.c_char_p
        L.drpt_last_error.restype = ctypes.c_char_p
        L.drpt_ctx_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int]
        L.drpt_ctx_destroy.argtypes = [vp]
        L.drpt_ctx_destroy.restype = None
        L.drpt_build_graph.argtypes = [vp, ctypes.POINTER(BuildDesc), vp, vp, vp,
                                       ctypes.POINTER(Stats)]
        L.drpt_build_graph_stream.argtypes = [vp, ctypes.POINTER(BuildDesc), i32,
                                              ctypes.POINTER(vp), ctypes.POINTER(vp),
                                              ctypes.POINTER(vp), ctypes.POINTER(Stats)]
        L.drpt_host_projection.argtypes = [u32, i32, i32, ctypes.c_float, vp]
        L.drpt_project.argtypes = [vp, vp, i64, i32, i32, vp, i32, vp, i32, vp, vp]
        L.drpt_project_sign.argtypes = [vp, vp, i64, i32, vp, i32, vp, i32, vp, vp]
        L.drpt_global_trees.argtypes = [vp, vp, i64, i32, i32, i32, vp, vp, vp, vp]
        L.drpt_local_leaves.argtypes = [vp, vp, vp, i64, i32, i32, i32, vp, vp, vp]
        L.drpt_locality_slots.argtypes = [vp, vp, i64, i32, i32, vp, vp, vp]
        L.drpt_leaf_knn.argtypes = [vp, vp, i32, i64, i32, i32, vp, vp, i32, i32, vp, vp, vp]
        L.drpt_merge_candidates.argtypes = [vp, vp, vp, i64, i32, i32, vp, vp, vp]
        L.drpt_global_trees_noalloc.argtypes = [vp, i64, i32, i32, i32, vp, vp, vp, vp]
        L.drpt_index_build.argtypes = [vp, ctypes.POINTER(BuildDesc), vp, vp, vp,
                                       ctypes.POINTER(Stats), ctypes.POINTER(vp)]
        L.drpt_index_query.argtypes = [vp, vp, i64, i32, i32, vp, vp, vp]
        L.drpt_index_destroy.argtypes = [vp]
        L.drpt_index_destroy.restype = None
        L.drpt_learn_gradient.argtypes = [vp, vp, i32, i32, vp, vp, vp, i32, vp, vp]
        L.drpt_build_graph_batched.argtypes = [vp, ctypes.POINTER(BatchDesc), vp, vp, vp, vp,
                                               ctypes.POINTER(Stats)]
        for name in EXPORTS:
            fn = getattr(L, name)
            if name not in ("drpt_version", "drpt_last_error", "drpt_ctx_destroy",
                            "drpt_index_destroy"):
                fn.restype = ctypes.c_int
        _lib = L
        return L


def check(status: int) -> None:
    if status != DRPT_OK:
        msg = load().drpt_last_error().decode(errors="replace")
        raise DrptError(status, msg)


class Context:
    """Owns a drpt_ctx (device workspace reused across calls)."""

    def __init__(self, device: int = 0):
        self._lib = load()
        self.handle = ctypes.c_void_p()
        check(self._lib.drpt_ctx_create(ctypes.byref(self.handle), device))
        self.device = device

    def close(self) -> None:
        if self.handle:
            self._lib.drpt_ctx_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_contexts: dict[int, Context] = {}


def context(device: int = 0) -> Context:
    ctx = _contexts.get(device)
    if ctx is None:
        ctx = _contexts[device] = Context(device)
    return ctx
