"""drpt_b200 -- the k-NN-graph path of DRPT (sparse random projection trees)
on NVIDIA B200 (sm_100a): hand-written CUDA kernels behind the C ABI of
libdrpt_gpu.so (include/drpt_gpu.h), a ctypes front end and the `drpt`
command line."""
from ._lib import DrptError, load as load_library  # noqa: F401
from .graph import (MDRPT, Index, build_graph, build_graph_batched,  # noqa: F401
                    build_graph_stream, build_index, edge_list_lines, global_depth)

__version__ = "0.1.0"
