"""The reference-side binding a maintainer would add (drpt_b200/adapter/,
shown in INTEGRATION.md): compiled against the reference's own headers
(drpt/algo/drpt_local.hpp for drpt::DataPoint) and linked with its
FileWriter (drpt/io/file_writer.cpp) by `make -C oracle adapter`, the driver
tests/adapter/adapter_main.cpp builds a graph through drpt_gpu_knn_graph and
writes the reference's edge list with the reference's writer.

CPU: the binding compiles in the reference tree and, without a GPU, the
library's failure reaches the caller as the exception the binding throws.
GPU: its results.txt equals the edge list of the same exact build made
through the Python API."""
import os
import subprocess

import numpy as np
import pytest

from drpt_b200 import build_graph, edge_list_lines, synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "adapter_check")


def _reference_root():
    root = os.environ.get("DRPT_REFERENCE_ROOT")
    if root and os.path.isdir(root):
        return root
    import __graft_entry__
    return __graft_entry__.REFERENCE_CHECKOUT if os.path.isdir(
        __graft_entry__.REFERENCE_CHECKOUT) else None


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except ImportError:
        return False


def test_binding_compiles_against_the_reference_headers(tmp_path):
    root = _reference_root()
    if root is None:
        pytest.skip("no reference checkout here (the binding is compiled where it is present)")
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "adapter",
                    "REF_ROOT=" + root], check=True)
    assert os.access(BIN, os.X_OK)
    if _has_gpu():
        return
    X = synth.clustered_f32(2_000, 16, n_clusters=20, seed=3)
    path = str(tmp_path / "x.fbin")
    synth.write_fbin(path, X)
    r = subprocess.run([BIN, path, str(tmp_path) + "/", "4", "10", "7"], capture_output=True,
                       text=True, timeout=120)
    # no device: drpt_ctx_create fails, the binding throws, the driver reports it
    assert r.returncode == 3, (r.returncode, r.stderr)
    assert "drpt_gpu_knn_graph:" in r.stderr


@pytest.mark.gpu
def test_binding_edge_list_equals_the_api_build(tmp_path):
    if not os.access(BIN, os.X_OK):
        pytest.skip("oracle/_ref/adapter_check was not built (no reference checkout at build)")
    X = synth.clustered_f32(12_000, 32, n_clusters=60, seed=9)
    path = str(tmp_path / "x.fbin")
    synth.write_fbin(path, X)
    r = subprocess.run([BIN, path, str(tmp_path) + "/", "6", "10", "4242"], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    got = open(tmp_path / "results.txt").read().split("\n")
    idx, _, _ = build_graph(X, 6, 10, 4242)
    want = edge_list_lines(np.asarray(idx), 9)
    assert [ln for ln in got if ln] == want
