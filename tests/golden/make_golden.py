"""Generates the golden fixtures in this directory by running the REFERENCE
itself (its own sources, built by `make -C oracle ref` with the one-rank MPI
stand-in, the ordered cblas and seed injection).

    python tests/golden/make_golden.py          # needs the reference tree

Each case_*.npz holds the seeded input, the run parameters and what the
reference produced: the projection matrix B, P = X.B, every tree's final
leaves (point ids in leaf order; P is omitted for the largest case plus leaf offsets, leaf ids in heap order with
-locality 0), the final leaves of the same run with -locality 1 (leaf ids in
the locality pass's slot order) and the first nn+4 entries of every point's merged neighbour
list exactly as gather_nns returned it (self and any duplicate entries
included).  median_cases.npz holds per-node means, variances and medians from
MathOp::distributed_mean/_variance/_median on hand-picked value sets,
including the degenerate ones (sigma = 0, n = 1, n = 0, the bin-14 tail).
"""
from __future__ import annotations

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

CASES = {
    # MNIST-shaped u8 data (config-1 distribution), fewer points.
    "u8_c1": dict(make=lambda: synth.clustered_u8(2000, 784, seed=11), ntrees=4, nn=10,
                  seeds=[12345, 1, 2, 3, 4]),
    # Gaussian clusters in float32 (config-2 distribution), fewer points and dims.
    "f32_c2": dict(make=lambda: synth.clustered_f32(16384, 32, n_clusters=400, seed=12), ntrees=8,
                   nn=10, seeds=[777] + list(range(11, 19)), keep_p=False),
    # Too few points per global leaf: the reference throws std::out_of_range
    # from DRPTLocal (local depth <= 0); the product must return its
    # depth-out-of-range status instead.
    "f32_depth_error": dict(make=lambda: synth.clustered_f32(4096, 32, n_clusters=40, seed=12),
                            ntrees=8, nn=10, seeds=[777] + list(range(11, 19)),
                            expect_error="out_of_range"),
    # A split sends every point of a node to one side, leaving a global leaf
    # empty; the reference throws from DRPTLocal (log2(0)); the product must
    # return its empty-leaf status.
    "f32_empty_leaf": dict(make=lambda: synth.clustered_f32(12000, 32, n_clusters=1000, seed=12),
                           ntrees=8, nn=10, seeds=[777] + list(range(11, 19)),
                           expect_error="out_of_range"),
    # Signed values, odd sizes, small nn.
    "f32_odd": dict(make=lambda: synth.clustered_f32(3001, 24, n_clusters=30, lo=-50.0, hi=50.0,
                                                     clip=None, seed=13), ntrees=5, nn=4,
                    seeds=[4242, 5, 6, 7, 8, 9]),
    # Small integer values: many exact distance ties and duplicate points.
    "u8_ties": dict(make=lambda: np.random.default_rng(14).integers(0, 4, size=(1500, 64))
                    .astype(np.uint8), ntrees=3, nn=6, seeds=[99, 1, 2, 3]),
}


def run_case(name: str, spec: dict, tmp: str) -> None:
    X = spec["make"]()
    n, d = X.shape
    is_u8 = X.dtype == np.uint8
    path = os.path.join(tmp, name + (".idx3" if is_u8 else ".fbin"))
    if is_u8:
        rows = 28 if d == 784 else 8
        synth.write_idx3(path, X, rows, d // rows)
    else:
        synth.write_fbin(path, X)
    dump0 = os.path.join(tmp, name + "_0.bin")
    if spec.get("expect_error"):
        try:
            refdump.run_reference(path, n, d, spec["ntrees"], spec["nn"], spec["seeds"],
                                  0 if is_u8 else 1, tmp, dump0, locality=0, dump_p=False)
        except RuntimeError as e:
            assert spec["expect_error"] in str(e), str(e)
            np.savez_compressed(os.path.join(HERE, f"case_{name}.npz"), X=X,
                                ntrees=spec["ntrees"], nn=spec["nn"],
                                seeds=np.asarray(spec["seeds"], np.uint32),
                                expect_error=spec["expect_error"], ref_stderr=str(e)[-300:])
            print(f"{name}: reference failed as expected ({spec['expect_error']})")
            return
        raise AssertionError(f"{name}: the reference was expected to fail")
    out = refdump.run_reference(path, n, d, spec["ntrees"], spec["nn"], spec["seeds"],
                                0 if is_u8 else 1, tmp, dump0, locality=0, dump_p=True)
    r = refdump.read(dump0)
    # The same run with the locality optimisation: at one rank it only
    # relabels leaves; record that the partition and the lists are unchanged.
    dump1 = os.path.join(tmp, name + "_1.bin")
    refdump.run_reference(path, n, d, spec["ntrees"], spec["nn"], spec["seeds"],
                          0 if is_u8 else 1, tmp, dump1, locality=1, dump_p=False)
    r1 = refdump.read(dump1)
    same_lists = all(np.array_equal(r["lists"][p][0], r1["lists"][p][0]) for p in range(n))

    def leafsets(rr):
        return [sorted(tuple(sorted(rr["final_order"][t, rr["final_offsets"][t, f]:
                                                       rr["final_offsets"][t, f + 1]].tolist()))
                       for f in range(rr["n_final"])) for t in range(rr["ntrees"])]

    same_partition = leafsets(r) == leafsets(r1)
    width = spec["nn"] + 4
    lidx = np.full((n, width), -1, np.int32)
    ldist = np.full((n, width), np.inf, np.float32)
    llen = np.zeros(n, np.int32)
    for p in range(n):
        li, ldd = r["lists"][p]
        llen[p] = len(li)
        lidx[p, :min(width, len(li))] = li[:width]
        ldist[p, :min(width, len(li))] = ldd[:width]
    edges = open(os.path.join(tmp, "results.txt")).read() if os.path.exists(
        os.path.join(tmp, "results.txt")) else ""
    np.savez_compressed(
        os.path.join(HERE, f"case_{name}.npz"), X=X, ntrees=spec["ntrees"], nn=spec["nn"],
        seeds=np.asarray(spec["seeds"], np.uint32), density=r["density"], gd=r["gd"], ld=r["ld"],
        n_final=r["n_final"], B=r["B"], P=r["P"] if spec.get("keep_p", True) else np.zeros(0, np.float32),
        final_order=r["final_order"],
        final_offsets=r["final_offsets"], list_idx=lidx, list_dist=ldist, list_len=llen,
        locality_same_partition=same_partition, locality_same_lists=same_lists,
        locality_final_order=r1["final_order"], locality_final_offsets=r1["final_offsets"],
        ref_stdout=out.strip().splitlines()[-1])
    print(f"{name}: n={n} d={d} gd={r['gd']} ld={r['ld']} n_final={r['n_final']} "
          f"locality partition/lists unchanged: {same_partition}/{same_lists} "
          f"edges={len(edges.splitlines())}")


def median_cases(tmp: str) -> None:
    rng = np.random.default_rng(21)
    nodes = [
        rng.normal(0.0, 1.0, 1000),                       # guard node (node 0 is never degenerate)
        rng.normal(5.0, 2.0, 777),
        rng.uniform(-10.0, 10.0, 500),
        rng.exponential(3.0, 999),
        np.full(50, 3.5),                                 # sigma = 0: every value lands in slot 0
        np.array([7.0]),                                  # n = 1: NaN variance, NaN median
        np.array([1.0, 2.0]),
        np.array([1.0, 2.0, 4.0]),
        np.concatenate([rng.normal(-100.0, 1.0, 90), np.full(10, -1.0)]),  # slot 14 tail
        1.0e6 + rng.normal(0.0, 0.01, 300),               # boundaries collapse in float
        np.concatenate([np.zeros(200), np.full(200, 100.0)]),
        rng.integers(0, 11, 640).astype(np.float64),      # values on boundaries, ties
        np.array([]),                                     # n = 0
        rng.normal(0.0, 1.0, 4097) * 1e-3,
        -rng.exponential(1.0, 333),
    ]
    sizes = np.array([len(v) for v in nodes], np.int32)
    vals = np.concatenate(nodes).astype(np.float32)
    inp = os.path.join(tmp, "median_in.bin")
    outp = os.path.join(tmp, "median_out.bin")
    with open(inp, "wb") as f:
        f.write(np.int32(len(nodes)).tobytes())
        f.write(sizes.tobytes())
        f.write(vals.tobytes())
    subprocess.run([os.path.join(ROOT, "oracle", "_ref", "drpt_ref"), "-median-test", inp, outp],
                   check=True)
    res = np.fromfile(outp, np.float32).reshape(3, len(nodes))
    np.savez_compressed(os.path.join(HERE, "median_cases.npz"), sizes=sizes, values=vals,
                        mean=res[0], var=res[1], median=res[2])
    print("median cases:", len(nodes))


def main() -> None:
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True)
    with tempfile.TemporaryDirectory() as tmp:
        median_cases(tmp)
        for name, spec in CASES.items():
            run_case(name, spec, tmp + "/")


if __name__ == "__main__":
    main()
