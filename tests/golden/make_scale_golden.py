"""Generates the two workload-sized parity fixtures in this directory by running
the REFERENCE itself (its own sources, built by `make -C oracle ref`; one rank,
one thread, seeds injected), at sizes too large for the fixtures of
make_golden.py to store whole:

* scale_c1_u8.npz -- the ubyte workload at its full size: 60,000 x 784 uint8
  (10 sparse centres, point spread sigma_p = 40), 8 trees, nn = 10,
  -locality 1.  (With the generator's default sigma_p = 20 every seed tried
  leaves a global leaf empty or too small and the reference stops with
  std::length_error in collect_similar_data_points; scale_c1_u8 records that
  too, for the error-status test.)
* scale_c2_f32.npz -- the fbin workload's distribution at 131,072 x 128
  float32 (131 Gaussian clusters, about 1,000 points each as at 1M), 16 trees,
  nn = 10, -locality 0.

Each holds the generator's parameters and the SHA-256 of the generated rows
(the tests regenerate them and check the hash first), the reference's depths,
the SHA-256 of every tree's final leaves (point ids in leaf order, and leaf
offsets), and its edge list (the first nn - 1 entries of every point's merged
list after dropping the point itself and repeated ids): whole as uint16 for
the 60,000-point case, as one 64-bit hash per point (plus every 32nd point's
ids) for the 131,072-point case.

    python tests/golden/make_scale_golden.py [--reuse DIR]

--reuse DIR reads the reference dumps DIR/scale_c1_u8.bin and
DIR/scale_c2_f32.bin and the stderr DIR/scale_c1_u8_sigma20.err of an earlier
run instead of running the reference again (about two and three minutes).
"""
from __future__ import annotations

import argparse
import hashlib
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from drpt_b200 import synth  # noqa: E402
from oracle import refdump  # noqa: E402
from tests import knn_compare  # noqa: E402

# Multiplier of the per-point edge-list hash (odd, 64-bit).
HASH_MUL = np.uint64(0x9E3779B97F4A7C15)

CASES = {
    "scale_c1_u8": dict(gen="clustered_u8", n=60_000, d=784, params=dict(sigma_p=40.0, seed=1),
                        ntrees=8, nn=10, seeds=[12345] + list(range(1, 9)), locality=1,
                        store="ids"),
    "scale_c2_f32": dict(gen="clustered_f32", n=131_072, d=128,
                         params=dict(n_clusters=131, seed=2), ntrees=16, nn=10,
                         seeds=[12345] + list(range(101, 117)), locality=0, store="hash"),
}


def make_rows(spec: dict) -> np.ndarray:
    return getattr(synth, spec["gen"])(spec["n"], spec["d"], **spec["params"])


def rows_sha(X: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(X).tobytes()).hexdigest()


def leaf_shas(order: np.ndarray, offsets: np.ndarray) -> np.ndarray:
    """One SHA-256 (hex) per tree over its int32 leaf order and offsets."""
    out = []
    for t in range(order.shape[0]):
        h = hashlib.sha256(np.ascontiguousarray(order[t], np.int32).tobytes())
        h.update(np.ascontiguousarray(offsets[t], np.int32).tobytes())
        out.append(h.hexdigest())
    return np.array(out)


def edge_hash(ids: np.ndarray) -> np.ndarray:
    """Per row, sum over j of (id_j + 1) * HASH_MUL^(j + 1) modulo 2^64."""
    ids = np.asarray(ids, np.int64)
    h = np.zeros(ids.shape[0], np.uint64)
    mul = np.uint64(1)
    with np.errstate(over="ignore"):
        for j in range(ids.shape[1]):
            mul = mul * HASH_MUL
            h = h + (ids[:, j] + 1).astype(np.uint64) * mul
    return h


def sigma20_error(tmp: str, reuse: str | None) -> str:
    """The reference on the ubyte workload's default spread (sigma_p = 20):
    its stderr tail, which names the exception it stops with."""
    if reuse:
        return open(os.path.join(reuse, "scale_c1_u8_sigma20.err")).read().strip()[-300:]
    X = synth.clustered_u8(60_000, 784, sigma_p=20.0, seed=1)
    path = os.path.join(tmp, "sigma20.idx3")
    synth.write_idx3(path, X, 28, 28)
    try:
        refdump.run_reference(path, 60_000, 784, 8, 10, [12345] + list(range(1, 9)), 0,
                              tmp + "/", os.path.join(tmp, "sigma20.bin"), locality=1,
                              dump_p=False)
    except RuntimeError as e:
        return str(e).strip()[-300:]
    raise AssertionError("the reference was expected to stop on the sigma_p = 20 rows")


def run_case(name: str, spec: dict, tmp: str, reuse: str | None, extra: dict) -> None:
    X = make_rows(spec)
    n, d = X.shape
    is_u8 = X.dtype == np.uint8
    dump = os.path.join(reuse, name + ".bin") if reuse else os.path.join(tmp, name + ".bin")
    if not reuse:
        path = os.path.join(tmp, name + (".idx3" if is_u8 else ".fbin"))
        if is_u8:
            synth.write_idx3(path, X, 28, 28)
        else:
            synth.write_fbin(path, X)
        refdump.run_reference(path, n, d, spec["ntrees"], spec["nn"], spec["seeds"],
                              0 if is_u8 else 1, tmp + "/", dump, locality=spec["locality"],
                              dump_p=False)
    r = refdump.read(dump)
    nn = spec["nn"]
    idx = np.full((n, nn + 3), -1, np.int32)
    dist = np.full((n, nn + 3), np.inf, np.float32)
    for p in range(n):
        li, ld = r["lists"][p]
        idx[p, :min(nn + 3, len(li))] = li[:nn + 3]
        dist[p, :min(nn + 3, len(ld))] = ld[:nn + 3]
    ri, _ = knn_compare.reference_first_k(idx, dist, nn - 1)
    out = dict(gen=spec["gen"], n=n, d=d, gen_params=repr(spec["params"]),
               rows_sha256=rows_sha(X), ntrees=spec["ntrees"], nn=nn,
               seeds=np.asarray(spec["seeds"], np.uint32), locality=spec["locality"],
               gd=r["gd"], ld=r["ld"], n_final=r["n_final"],
               leaf_sha256=leaf_shas(r["final_order"], r["final_offsets"]), **extra)
    if spec["store"] == "ids":
        assert n <= 65535
        out["edge_ids"] = ri.astype(np.uint16)
    else:
        out["edge_hash"] = edge_hash(ri)
        out["sample_points"] = np.arange(0, n, 32, dtype=np.int32)
        out["sample_edge_ids"] = ri[::32].astype(np.int32)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(f"{name}: n={n} d={d} gd={r['gd']} ld={r['ld']} n_final={r['n_final']}")


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reuse", default=None)
    args = ap.parse_args()
    if not args.reuse:
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True)
    with tempfile.TemporaryDirectory(dir=os.path.join(ROOT, "oracle", "_ref")) as tmp:
        err = sigma20_error(tmp, args.reuse)
        assert "length_error" in err, err
        for name, spec in CASES.items():
            extra = {"sigma20_reference_error": err} if name == "scale_c1_u8" else {}
            run_case(name, spec, tmp, args.reuse, extra)


if __name__ == "__main__":
    main()
