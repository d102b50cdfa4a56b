"""Reader for the binary dump written by the reference driver
(oracle/refbuild/ref_driver.cpp, ``-dump``).  Test infrastructure only.

Layout (little-endian): b"DRPTREF1"; int32 n, d, ntrees, nn, gd, ld, n_final,
has_p; float64 density; float32 B[d][gd*ntrees]; float32 P[n][gd*ntrees] when
has_p; for each tree, for each final leaf id: int32 size, int32 index[size];
int32 n_lists; per list: int32 point, int32 count, count x (int32 index,
float32 distance).
"""
from __future__ import annotations

import os
import subprocess

import numpy as np


def read(path: str) -> dict:
    buf = open(path, "rb").read()
    assert buf[:8] == b"DRPTREF1", "not a reference dump"
    pos = 8
    hdr = np.frombuffer(buf, np.int32, 8, pos)
    pos += 32
    n, d, T, nn, gd, ld, nfinal, has_p = (int(v) for v in hdr)
    density = float(np.frombuffer(buf, np.float64, 1, pos)[0])
    pos += 8
    L = gd * T
    B = np.frombuffer(buf, np.float32, d * L, pos).reshape(d, L).copy()
    pos += 4 * d * L
    P = None
    if has_p:
        P = np.frombuffer(buf, np.float32, n * L, pos).reshape(n, L).copy()
        pos += 4 * n * L
    order = np.empty((T, n), np.int32)
    offsets = np.empty((T, nfinal + 1), np.int32)
    for t in range(T):
        w = 0
        for f in range(nfinal):
            sz = int(np.frombuffer(buf, np.int32, 1, pos)[0])
            pos += 4
            offsets[t, f] = w
            order[t, w:w + sz] = np.frombuffer(buf, np.int32, sz, pos)
            pos += 4 * sz
            w += sz
        offsets[t, nfinal] = w
    nl = int(np.frombuffer(buf, np.int32, 1, pos)[0])
    pos += 4
    lists = {}
    for _ in range(nl):
        p, c = (int(v) for v in np.frombuffer(buf, np.int32, 2, pos))
        pos += 8
        rec = np.frombuffer(buf, dtype=[("idx", "<i4"), ("dist", "<f4")], count=c, offset=pos)
        pos += 8 * c
        lists[p] = (rec["idx"].copy(), rec["dist"].copy())
    return {"n": n, "d": d, "ntrees": T, "nn": nn, "gd": gd, "ld": ld, "n_final": nfinal,
            "density": density, "B": B, "P": P, "final_order": order, "final_offsets": offsets,
            "lists": lists}


def run_reference(input_path: str, n: int, d: int, ntrees: int, nn: int, seeds, fmt: int,
                  out_dir: str, dump_path: str, locality: int = 0, dump_p: bool = True,
                  threads: int = 1, ref_bin: str | None = None, extra=()):
    """Run the reference binary (oracle/_ref/drpt_ref) once.  Returns its
    stdout.  `seeds` = [global seed, local seed per tree...]."""
    here = os.path.dirname(os.path.abspath(__file__))
    ref_bin = ref_bin or os.path.join(here, "_ref", "drpt_ref")
    env = dict(os.environ)
    env["DRPT_REF_SEEDS"] = ",".join(str(int(s) & 0xFFFFFFFF) for s in seeds)
    env["OMP_NUM_THREADS"] = str(threads)
    args = [ref_bin, "-input", input_path, "-output", out_dir.rstrip("/") + "/",
            "-data-set-size", str(n), "-dimension", str(d), "-ntrees", str(ntrees), "-nn", str(nn),
            "-locality", str(locality), "-data-file-format", str(fmt), "-dump", dump_path]
    if dump_p:
        args.append("-dump-p")
    args += list(extra)
    cmd = "ulimit -s unlimited; exec " + " ".join(subprocess.list2cmdline([a]) for a in args)
    r = subprocess.run(["bash", "-c", cmd], env=env, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"reference run failed ({r.returncode}): {r.stderr[-2000:]}")
    return r.stdout


def first_k_non_self(lists: dict, n: int, k: int):
    """The reference's merged lists cut to each point's first k entries that
    are not the point itself (what the edge-list writer keeps with k = nn-1,
    file_writer.cpp:95-99).  Pads with -1 / inf."""
    idx = np.full((n, k), -1, np.int64)
    dist = np.full((n, k), np.inf, np.float32)
    for p in range(n):
        li, ld = lists[p]
        keep = li != p
        li, ld = li[keep][:k], ld[keep][:k]
        idx[p, :len(li)] = li
        dist[p, :len(ld)] = ld
    return idx, dist
