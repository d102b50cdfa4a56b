"""The `drpt` command-line program: the reference CLI's flags, checks, input
formats, edge-list file and timing line (cpp/src/main.cpp)."""
import gzip
import os
import shutil
import struct
import subprocess

import numpy as np
import pytest

from drpt_b200 import build, build_graph, edge_list_lines, synth
from tests import knn_compare
from tests.conftest import GOLDEN


@pytest.fixture(scope="module")
def cli():
    path = build.build_cli()
    if not path:
        pytest.fail("the drpt CLI did not build")
    return path


def _run(cli, *args, timeout=300):
    return subprocess.run([cli, *map(str, args)], capture_output=True, text=True, timeout=timeout)


@pytest.mark.parametrize("drop,message", [
    ("-input", "Valid input path needed!..."),
    ("-output", "Valid out path needed!..."),
    ("-data-set-size", "Dataset size should be greater than 0"),
    ("-dimension", "Dimension size should be greater than 0"),
    ("-nn", "Nearest neighbours size should be greater than 0"),
])
def test_required_flags(cli, tmp_path, drop, message):
    flags = {"-input": "x.bin", "-output": str(tmp_path) + "/", "-data-set-size": 100,
             "-dimension": 8, "-nn": 5}
    del flags[drop]
    args = [a for kv in flags.items() for a in kv]
    r = _run(cli, *args)
    assert r.returncode == 1 and r.stdout.strip() == message


def test_unsupported_format_and_short_files(cli, tmp_path):
    x = np.arange(64 * 16, dtype=np.float32).reshape(64, 16)
    fb = tmp_path / "x.fbin"
    synth.write_fbin(str(fb), x)
    base = ["-input", fb, "-output", str(tmp_path) + "/", "-dimension", 16, "-nn", 4]
    r = _run(cli, *base, "-data-set-size", 64, "-data-file-format", 2)
    assert r.returncode == 1 and "Unsupported data file format" in r.stdout
    r = _run(cli, *base, "-data-set-size", 65, "-data-file-format", 1)
    assert r.returncode == 1 and "fewer points" in r.stdout  # the header holds 64
    short = tmp_path / "short.fbin"
    with open(short, "wb") as f:  # header claims 65 points, the file holds 64
        f.write(struct.pack("<II", 65, 16) + x.tobytes())
    r = _run(cli, "-input", short, "-output", str(tmp_path) + "/", "-dimension", 16, "-nn", 4,
             "-data-set-size", 65, "-data-file-format", 1)
    assert r.returncode == 1 and "fewer than" in r.stdout
    ub = tmp_path / "x.idx3"
    synth.write_idx3(str(ub), np.zeros((10, 16), np.uint8), rows=4, cols=4)
    r = _run(cli, "-input", ub, "-output", str(tmp_path) + "/", "-dimension", 16, "-nn", 4,
             "-data-set-size", 11)
    assert r.returncode == 1 and "fewer images" in r.stdout
    r = _run(cli, "-input", ub, "-output", str(tmp_path) + "/", "-dimension", 15, "-nn", 4,
             "-data-set-size", 10)
    assert r.returncode == 1 and "-dimension" in r.stdout


def _parse_edges(path, n, per_point):
    idx = np.full((n, per_point), -1, np.int64)
    fill = np.zeros(n, np.int64)
    with open(path) as f:
        for line in f:
            s, t = line.split()
            s = int(s) - 1
            idx[s, fill[s]] = int(t) - 1
            fill[s] += 1
    return idx


@pytest.mark.gpu
@pytest.mark.parametrize("case,fmt", [("case_u8_c1", 0), ("case_f32_odd", 1)])
def test_cli_graph_matches_reference(cli, tmp_path, case, fmt):
    g = np.load(os.path.join(GOLDEN, case + ".npz"))
    X = g["X"]
    n, d = X.shape
    T, nn = int(g["ntrees"]), int(g["nn"])
    seed = int(g["seeds"][0])
    if fmt == 0:
        path = tmp_path / "data.idx3"
        synth.write_idx3(str(path), X, rows=28, cols=28)
        extra = []
    else:
        path = tmp_path / "data.fbin"
        synth.write_fbin(str(path), X)
        extra = ["-data-file-format", 1, "-bytes-for-data-type", 4, "-data-starting-index", 8]
    out = str(tmp_path) + "/"
    r = _run(cli, "-input", path, "-output", out, "-data-set-size", n, "-dimension", d,
             "-ntrees", T, "-nn", nn, "-seed", seed, *extra)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "IO Time (s)" in r.stdout and "Index building (s)" in r.stdout
    with open(out + "results.txt") as f:
        text = f.read()
    # identical to the library call on the same inputs
    idx, _, _ = build_graph(X, T, nn, seed)
    assert text == "".join(line + "\n" for line in edge_list_lines(idx, nn - 1))
    # and to the reference's edge list up to exact-distance ties
    ri, rd = knn_compare.reference_first_k(g["list_idx"], g["list_dist"], nn + 3)
    got = _parse_edges(out + "results.txt", n, nn - 1)
    _, dist, _ = build_graph(X, T, nn, seed)
    res = knn_compare.compare(ri[:, :nn - 1], rd[:, :nn - 1], got, dist[:, :nn - 1], rd)
    assert res["fail"] == 0, res
    assert os.path.getsize(out + "stats.txt") > 0
    # -locality 1 renumbers the global leaves only: the same edge list
    out1 = str(tmp_path / "loc") + "/"
    os.makedirs(out1)
    r = _run(cli, "-input", path, "-output", out1, "-data-set-size", n, "-dimension", d,
             "-ntrees", T, "-nn", nn, "-seed", seed, "-locality", 1, *extra)
    assert r.returncode == 0, r.stdout + r.stderr
    with open(out1 + "results.txt") as f:
        assert f.read() == text


def test_header_checks(cli, tmp_path):
    """IDX3 magic and fbin header are checked against the flags."""
    out = str(tmp_path) + "/"
    bad = tmp_path / "bad.idx3"
    with open(bad, "wb") as f:
        f.write(struct.pack(">iiii", 0x0801, 10, 4, 4) + bytes(160))
    r = _run(cli, "-input", bad, "-output", out, "-dimension", 16, "-nn", 4, "-data-set-size", 10)
    assert r.returncode == 1 and "magic" in r.stdout
    fb = tmp_path / "x.fbin"
    synth.write_fbin(str(fb), np.zeros((64, 16), np.float32))
    base = ["-input", fb, "-output", out, "-nn", 4, "-data-file-format", 1]
    r = _run(cli, *base, "-dimension", 8, "-data-set-size", 64)  # 16-wide rows, 8 claimed
    assert r.returncode == 1 and "dimension" in r.stdout
    big = tmp_path / "big.fbin"
    with open(big, "wb") as f:  # header says 32 points, the file holds 64
        f.write(struct.pack("<II", 32, 16) + np.zeros((64, 16), np.float32).tobytes())
    r = _run(cli, "-input", big, "-output", out, "-nn", 4, "-data-file-format", 1,
             "-dimension", 16, "-data-set-size", 64)
    assert r.returncode == 1 and "fewer points" in r.stdout


@pytest.mark.gpu
def test_cli_gzip_input_and_distance_column(cli, tmp_path):
    """A gzip-compressed IDX3 file gives the same edge list as the plain one;
    -write-distances adds each edge's FP32 distance."""
    g = np.load(os.path.join(GOLDEN, "case_u8_c1.npz"))
    X = g["X"]
    n, d = X.shape
    T, nn, seed = int(g["ntrees"]), int(g["nn"]), int(g["seeds"][0])
    plain = tmp_path / "data.idx3"
    synth.write_idx3(str(plain), X, rows=28, cols=28)
    packed = tmp_path / "data.idx3.gz"
    with open(plain, "rb") as fi, gzip.open(packed, "wb") as fo:
        shutil.copyfileobj(fi, fo)
    texts = []
    for path, extra in ((plain, []), (packed, []), (packed, ["-write-distances", 1])):
        out = tmp_path / f"o{len(texts)}"
        out.mkdir()
        r = _run(cli, "-input", path, "-output", str(out) + "/", "-data-set-size", n,
                 "-dimension", d, "-ntrees", T, "-nn", nn, "-seed", seed, *extra)
        assert r.returncode == 0, r.stdout + r.stderr
        texts.append(open(out / "results.txt").read())
    assert texts[0] == texts[1]
    _, dist, _ = build_graph(X, T, nn, seed)
    rows = [line.split() for line in texts[2].splitlines()]
    assert [r[:2] for r in rows] == [line.split() for line in texts[0].splitlines()]
    seen = {}
    for src, dst, dv in rows:
        p = int(src) - 1
        j = seen.get(p, 0)
        seen[p] = j + 1
        assert float(dv) == pytest.approx(float(dist[p, j]), rel=1e-7)
