"""Benchmark of the k-NN-graph path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--mode mixed|exact|fast]
                    [--impl ours|reference]

Workload (one step = one complete graph build of 1,000,000 x 128 float32
points, a mixture of 1,000 Gaussian clusters with centres U[0,200]^128,
sigma 12, clipped to [0,255]; nn = 10; synthetic data of the shape of the
fbin workload).  The headline form is the mixed-precision one (6 trees,
global leaves of about 1,024 points, BF16 tensor-core leaf tiles, exact FP32
re-rank), which reaches recall@10 >= 0.90; beside it, at one GPU, the plain
FP32 form with the reference's parameters (16 trees, reference-exact) and the
plain form with enough trees to approach the same recall are timed once.
`value` is points/s with the input resident in HBM (512 MB, larger than L2,
so no flush is needed between steps); `e2e` is the same build through the
public host-pointer call with the input copied from pinned host memory and
the neighbour lists copied back, every step.

Under torchrun (N > 1) every rank builds an independent graph of its own
1M-point dataset (the path has no inter-GPU exchange: replicas, weak
scaling); the step time is the maximum over ranks.

--impl reference times the reference's own CPU implementation (the reference
sources built by `make -C oracle ref`, 1 rank x all host threads) on a
bounded sample of the same workload.

--workload picks one of the other k-NN-graph workloads (one GPU; the same
JSON line, with the mixed form's equal-recall FP32 counterpart beside it):
  ubyte-60k-784   60,000 x 784 uint8 (IDX3-shaped), 10 sparse centres, nn 10
  fbin-2m-960     2,000,000 x 960 float32, 500 anisotropic Gaussians in
                  [0,1], nn 20, FP8-E4M3 leaf tiles (BF16 beside)
  batch-256x96    256 float32 datasets of 96 dims, sizes log-uniform in
                  [2,000, 200,000], nn 16, one batched build replayed from a
                  CUDA graph
  learned-1m-256  1,000,000 x 256 float32 on a 16-dim latent manifold, nn 10,
                  8 random + 8 learned trees beside 16 and 32 random trees
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "kNN-graph points/s at recall@10≥0.90, mixed/learned vs plain FP32, 1 B200"
N_POINTS, DIM, NTREES, NN, N_CLUSTERS = 1_000_000, 128, 16, 10, 1000
MIXED_TREES, MIXED_LEAF = 6, 1024   # mixed form: trees and target global-leaf size
PLAIN_MATCH_TREES = 384             # the reference method with many more trees
SEED_PROJ = 12345
CPU_SAMPLE = 32_768  # bounded sample for the CPU baseline (about 10-30 s of CPU work)
# Samples of --impl reference, timed and untimed steps: the size of the CPU
# baseline's sample.  On some smaller samples of this distribution (4,096,
# 8,192 and 16,384 points among them) the reference's smallest global leaf is
# too small for its local trees and it throws std::out_of_range.
REF_STEP_SAMPLE = 32_768
REF_WARMUP_SAMPLE = 32_768
WORKLOAD = ("1,000,000 x 128 float32 (fbin-shaped), 1000 Gaussian clusters, centres U[0,200]^128, "
            "sigma 12, clipped to [0,255]; nn=10")
# Tree parameters of each arm.  The metric is points/s at recall@10 >= 0.90:
# the mixed form's trees are chosen for that recall.  The reference's own
# parameters (16 trees, positional local split) give a recall that depends on
# its thread count: at one thread every node lists its points in index order
# and the positional chunks of all trees repeat the same neighbours (recall@10
# 0.55 on the 32,768-point sample, 0.10 at 1M points, the order the exact
# form reproduces); with many threads the order inside a node varies per tree
# and recall rises (0.96 on the same sample at 8 threads).  The reference arm
# reports the recall of the run it timed.
TREES_MIXED = (f"mixed form: {MIXED_TREES} trees, global leaves of about {MIXED_LEAF} points "
               "brute-forced whole (chosen for recall@10 >= 0.90)")
TREES_REFERENCE = (f"reference parameters: {NTREES} trees, tree depth int(log2 n - 2), ratio 0.6, "
                   "positional local split")
# The reference's cblas calls (sgemm of the projection, saxpy/snrm2 of its
# distance) run in OpenBLAS, the library its build names: numpy's bundled
# scipy-openblas (oracle/_ref/drpt_ref_openblas, `make -C oracle
# ref-openblas`).  Without that build they run in the project's ordered cblas
# (plain loops in a fixed summation order, oracle/refbuild/cblas_ordered.cpp),
# the build the parity tests use.
REF_BINARIES = (("drpt_ref_openblas", "OpenBLAS (numpy's bundled scipy-openblas, "
                 "oracle/refbuild/cblas_openblas.cpp)"),
                ("drpt_ref", "ordered cblas (plain loops, oracle/refbuild/cblas_ordered.cpp)"))


def _reference_cblas() -> str:
    found = _reference_binary()
    return found[1] if found else "none (the CPU restatement was timed)"


def _loads(path: str) -> bool:
    """True unless the dynamic loader reports a missing library for `path`."""
    try:
        r = subprocess.run(["ldd", path], capture_output=True, text=True, timeout=30)
    except (OSError, subprocess.SubprocessError):
        return True  # no ldd: let the run itself report a failure
    return "not found" not in r.stdout


def _reference_binary():
    """(path, cblas description) of the reference build to time, or None:
    the OpenBLAS build where its library loads, else the ordered-cblas one."""
    for name, cblas in REF_BINARIES:
        path = os.path.join(ROOT, "oracle", "_ref", name)
        if os.path.exists(path) and _loads(path):
            return path, cblas
    return None


def _env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def _cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), parts[4:9]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for _, _, r in rows:
            for nm, v in zip(names, r[1:]):
                if v.lower() == "active":
                    reasons.add(nm)
        sm = [r[0] for r in rows]
        loaded = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": max(r[1] for r in rows),
                "samples": len(rows), "reasons": sorted(reasons)}


# ---------------------------------------------------------------- reference arm
def _reference_sample(tmpdir: str, n: int):
    from drpt_b200 import synth
    X = synth.clustered_f32(n, DIM, n_clusters=max(1, round(N_CLUSTERS * n / N_POINTS)), seed=2)
    path = os.path.join(tmpdir, "sample.fbin")
    synth.write_fbin(path, X)
    return X, path


def run_reference_once(path: str, n: int, threads: int, dump: str | None = None):
    """One run of the reference binary; returns (build_s, query_s, kind).
    `dump`: a file for its merged neighbour lists (written after the timed
    phases)."""
    found = _reference_binary()
    seeds = ",".join(str(s) for s in [SEED_PROJ] + list(range(1, NTREES + 1)))
    if found:
        ref = found[0]
        out_dir = tempfile.mkdtemp()
        cmd = (f"ulimit -s unlimited; exec {ref} -input {path} -output {out_dir}/ -data-set-size {n} "
               f"-dimension {DIM} -ntrees {NTREES} -nn {NN} -locality 0 -data-file-format 1 -no-write"
               + (f" -dump {dump}" if dump else ""))
        env = dict(os.environ, DRPT_REF_SEEDS=seeds, OMP_NUM_THREADS=str(threads),
                   OPENBLAS_NUM_THREADS=str(threads), OMP_PROC_BIND="true")
        r = subprocess.run(["bash", "-c", cmd], env=env, capture_output=True, text=True)
        shutil.rmtree(out_dir, ignore_errors=True)
        m = re.search(r"Index building \(s\)\s*([0-9.eE+-]+)\s*Querying Time \(s\)\s*([0-9.eE+-]+)",
                      r.stdout)
        if r.returncode != 0 or not m:
            raise RuntimeError(f"reference run failed: {r.stderr[-500:]}")
        return float(m.group(1)), float(m.group(2)), "reference"
    # The reference tree was not built here: time the CPU restatement instead.
    import oracle
    from drpt_b200 import synth
    X = synth.read_fbin(path)
    t0 = time.perf_counter()
    o = oracle.build(X, NTREES, NN, SEED_PROJ)
    t1 = time.perf_counter()
    if o["status"] != 0:
        raise RuntimeError(f"oracle build failed: {o['status']}")
    return t1 - t0, 0.0, "port"


def reference_recall(X, dump: str, queries: int = 1000) -> float:
    """recall@10 of the reference's merged lists (each point's first nn = 10
    non-self candidates; the edge list it writes holds the first 9) against
    FP64 exact neighbours of a seeded sample, by the CPU checker."""
    import oracle
    from oracle import refdump
    from drpt_b200 import recall
    lists = refdump.read(dump)["lists"]
    n = len(X)
    idx, _ = refdump.first_k_non_self(lists, n, NN)
    q = recall.sample_queries(n, queries, seed=7)
    ti, _ = oracle.exact_knn(X, q, NN)
    return recall.recall_at_k(idx[q], ti)


def cpu_baseline(n: int = CPU_SAMPLE):
    threads = _cores()
    with tempfile.TemporaryDirectory() as tmp:
        X, path = _reference_sample(tmp, n)
        dump = os.path.join(tmp, "lists.bin")
        b, q, kind = run_reference_once(path, n, threads, dump=dump)
        rec = reference_recall(X, dump) if kind == "reference" else None
    return {"value": n / (b + q), "unit": "points/s", "cores": threads if kind == "reference" else 1,
            "kind": kind,
            "sample": f"{n} points of the same distribution (clusters scaled to {max(1, round(N_CLUSTERS * n / N_POINTS))}), "
                      f"{TREES_REFERENCE}, nn={NN}, 1 rank x {threads if kind == 'reference' else 1} threads; "
                      f"time = index building + querying ({b:.2f} s + {q:.2f} s); "
                      f"cblas: {_reference_cblas()}",
            "recall@10": rec}


def reference_arm(args):
    rank = _env_int("RANK", 0)
    if rank != 0:
        return
    threads = _cores()
    times = []
    rec = None
    with tempfile.TemporaryDirectory() as tmp:
        _, wpath = _reference_sample(tmp, REF_WARMUP_SAMPLE)
        for _ in range(args.warmup):
            run_reference_once(wpath, REF_WARMUP_SAMPLE, threads)
        X, path = _reference_sample(tmp, REF_STEP_SAMPLE)
        kind = "reference"
        for _ in range(args.steps):
            b, q, kind = run_reference_once(path, REF_STEP_SAMPLE, threads)
            times.append(b + q)
        if kind == "reference":
            # quality of what was timed: one more untimed run dumps its lists
            dump = os.path.join(tmp, "lists.bin")
            run_reference_once(path, REF_STEP_SAMPLE, threads, dump=dump)
            rec = reference_recall(X, dump)
    sec = sum(times) / len(times)
    value = REF_STEP_SAMPLE / sec
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "points/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "trees": TREES_REFERENCE, "ntrees": NTREES,
                   "sample_points": REF_STEP_SAMPLE, "ranks": 1, "threads": threads,
                   "recall@10": rec, "recall_sample": 1000, "cblas": _reference_cblas(),
                   "note": "the sample is bounded so that the run ends in minutes; the "
                           "reference's recall depends on its thread count (the order of "
                           "points inside a node feeds its positional local split)"},
        "cpu_baseline": {"value": value, "unit": "points/s", "cores": threads if kind == "reference" else 1,
                         "kind": kind,
                         "sample": f"{REF_STEP_SAMPLE} points of the same distribution per timed step "
                                   f"(warm-up steps: {REF_WARMUP_SAMPLE} points)"},
        "e2e": {"value": value, "unit": "points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)



# ---------------------------------------------------------------- other workloads
def _timed(fn, steps):
    """Mean device time (ms) of `steps` calls of fn after one untimed call,
    CUDA events on the current stream; returns (last result, ms)."""
    import torch
    out = fn()
    torch.cuda.synchronize()
    s = torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(s)
    for _ in range(steps):
        out = fn()
    b.record(s)
    torch.cuda.synchronize()
    return out, a.elapsed_time(b) / steps


def other_workload(args):
    import torch

    from drpt_b200 import build_graph, build_graph_batched, recall, synth
    if _env_int("RANK", 0) != 0:
        return
    torch.cuda.set_device(0)
    steps, warm = args.steps, max(args.warmup, 3)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    wl = args.workload
    comps = {}

    def rec_of(idx, q, ti, k):
        return recall.recall_at_k(idx.cpu().numpy()[q][:, :k], ti[:, :k])

    if wl == "batch-256x96":
        sizes = synth.batch_sizes(256, 2_000, 200_000, seed=4)
        sets = [synth.batch_dataset(int(m), 96, seed=1000 + i) for i, m in enumerate(sizes)]
        offs = np.concatenate([[0], np.cumsum([len(x) for x in sets])]).astype(np.int64)
        X = np.concatenate(sets)
        n, d, nn, T = len(X), 96, 16, 8
        Xd = torch.from_numpy(X).cuda()
        idx = torch.empty((n, nn), dtype=torch.int32, device="cuda")
        dst = torch.empty((n, nn), dtype=torch.float32, device="cuda")

        # leaf size and list width picked by the autotuner on this batch
        # (outside the timed region; its trials are reported)
        from drpt_b200 import autotune
        tuned = autotune.tune_batched(Xd, offs, T, nn, SEED_PROJ, target_recall=0.90,
                                      leaf_sizes=(256, 512, 1024), reps=1)
        leaf, width = tuned["leaf_size"], tuned["list_width"]

        def run():
            return build_graph_batched(Xd, offs, T, nn, SEED_PROJ, mode="mixed", leaf_size=leaf,
                                       use_graph=True, out=(idx, dst), list_width=width)[2]
        for _ in range(warm):
            run()
        with ClockSampler(0) as clocks:
            st, ms = _timed(run, steps)
        clk = clocks.summary()
        recs = []
        for s in range(0, 256, 32):  # every 32nd dataset, 100 queries each
            x = sets[s]
            q = recall.sample_queries(len(x), 100, seed=s)
            ti, _ = recall.exact_knn_fp64(x, q, 10)
            recs.append(recall.recall_at_k(idx[offs[s]:offs[s + 1]].cpu().numpy()[q][:, :10], ti))
        rec = float(np.mean(recs))
        (i32, _, st32), ms32 = _timed(lambda: build_graph_batched(Xd, offs, T, nn, SEED_PROJ,
                                                                  mode="fp32_leaf",
                                                                  leaf_size=leaf), 1)
        recs32 = []
        for s in range(0, 256, 32):
            q = recall.sample_queries(len(sets[s]), 100, seed=s)
            ti, _ = recall.exact_knn_fp64(sets[s], q, 10)
            recs32.append(recall.recall_at_k(np.asarray(i32[offs[s]:offs[s + 1]].cpu())[q][:, :10],
                                             ti))
        comps["fp32_leaf_batched_same_trees"] = {"points_per_s": n / (ms32 / 1e3), "ms": ms32,
                                                 "recall@10": float(np.mean(recs32))}
        comps["mixed_over_plain_fp32_at_equal_recall"] = ms32 / ms
        cfg = {"workload": "256 float32 datasets, d=96, sizes log-uniform [2000, 200000] "
                           f"({n} points), 20-200 Gaussians each (sigma 1, centres U[-10,10]); nn=16",
               "mode": "mixed, batched, CUDA-graph replay", "ntrees": T, "leaf_size": leaf,
               "list_width": width, "recall@10": rec,
               "recall_sample": "100 queries in each of 8 datasets",
               "kernels_per_build": st.kernels_launched,
               "autotune": {"target_recall@10": 0.90, "tune_s": round(tuned["tune_s"], 2),
                            "trials": tuned["trials"],
                            "note": "leaf size x list width measured on this batch before "
                                    "the timed region (50 queries in each of 8 datasets)"}}
        launches = st.kernels_launched * steps
        roof = None
    else:
        # --points: a smaller case of the same distribution, for profiling only
        pts = args.points
        if wl == "ubyte-60k-784":
            X = synth.clustered_u8(pts or 60_000, 784, seed=1)
            nn, T, leaf, prec, lt = 10, 12, 1024, "bf16", 0
            desc = "60,000 x 784 uint8 (IDX3-shaped), 10 centres with 80% zero coordinates, sigma 20"
        elif wl == "fbin-2m-960":
            X = synth.anisotropic_f32(pts or 2_000_000, 960,
                                      n_clusters=max(1, round(500 * (pts or 2_000_000) / 2e6)),
                                      seed=3)
            nn, T, leaf, prec, lt = 20, 32, 2048, "fp8", 0
            desc = ("2,000,000 x 960 float32, 500 anisotropic Gaussians (per-dim sigma U[0.01,0.3]), "
                    "values in [0,1]")
        else:
            X = synth.latent_manifold_f32(pts or 1_000_000, 256, seed=5)
            nn, T, leaf, prec, lt = 10, 16, 1024, "bf16", 8
            desc = "1,000,000 x 256 float32, x = tanh(A z + b) * 4 + N(0, 0.05^2), z ~ N(0, I_16)"
        if pts:
            desc = f"{pts:,}-point profiling case of: " + desc
        n, d = X.shape
        Xd = torch.from_numpy(X).cuda()
        del X
        idx = torch.empty((n, nn), dtype=torch.int32, device="cuda")
        dst = torch.empty((n, nn), dtype=torch.float32, device="cuda")

        # config 5 trains the split MLPs on a 50k-point sample; 3 Adam steps per
        # level (recall 0.840 against 0.844 with 10 steps, at half the training)
        sample, iters = (50_000, 3) if lt else (0, 0)

        def run(mode="mixed", trees=T, precision=prec, learned=lt, out=(idx, dst), smp=sample,
                projection="gaussian"):
            return build_graph(Xd, trees, nn, SEED_PROJ, mode=mode, leaf_size=leaf,
                               precision=precision, learned_trees=learned, out=out,
                               learn_sample=smp if learned else 0,
                               learn_iters=iters if learned else 0, projection=projection)[2]
        for _ in range(warm):
            run()
        with ClockSampler(0) as clocks:
            st, ms = _timed(run, steps)
        clk = clocks.summary()
        q = recall.sample_queries(n, 300 if d > 512 else 1000, seed=7)
        ti, _ = recall.exact_knn_fp64(Xd, q, nn)
        rec = rec_of(idx, q, ti, 10)
        cfg = {"workload": desc + f"; nn={nn}", "mode": "mixed", "precision": prec, "ntrees": T,
               "learned_trees": lt, "leaf_size": leaf, "recall@10": rec,
               f"recall@{nn}": rec_of(idx, q, ti, nn), "recall_sample": len(q),
               "phase_ms": {k: getattr(st, "ms_" + k) for k in
                            ("global", "leaf_knn", "merge", "leaf_mma", "leaf_stage", "learn")}}
        if lt:
            cfg["learn_loss"] = [st.learn_loss_start, st.learn_loss_end]
        launches = st.kernels_launched * steps
        pi = torch.empty_like(idx)
        pd = torch.empty_like(dst)
        others = []
        if wl == "fbin-2m-960":
            others.append(("mixed_bf16", dict(precision="bf16")))
        if wl == "ubyte-60k-784":
            # the u8 rows projected with the sign matrix on the tensor cores
            others.append(("mixed_sign_projection", dict(projection="sign")))
        if lt:
            others += [("mixed_learned_sample_8192", dict(smp=8192)),
                       (f"mixed_{T}_random_trees", dict(learned=0)),
                       (f"mixed_{2 * T}_random_trees", dict(trees=2 * T, learned=0)),
                       # a learned configuration past recall 0.90, and random
                       # trees to meet it
                       (f"mixed_{T}_random_{T}_learned_trees", dict(trees=2 * T, learned=T)),
                       (f"mixed_{3 * T}_random_trees", dict(trees=3 * T, learned=0)),
                       (f"fp32_leaf_{2 * T}_random_trees", dict(mode="fp32_leaf", trees=2 * T,
                                                                  learned=0)),
                       (f"fp32_gram_{2 * T}_random_trees", dict(mode="fp32_gram", trees=2 * T,
                                                                  learned=0))]
        else:
            others.append((f"fp32_leaf_{T}_trees", dict(mode="fp32_leaf")))
            others.append((f"fp32_gram_{T}_trees", dict(mode="fp32_gram")))
        for name, kw in others:
            pst, pms = _timed(lambda: run(out=(pi, pd), **kw), 1)
            comps[name] = {"points_per_s": n / (pms / 1e3), "ms": pms,
                           "recall@10": rec_of(pi, q, ti, 10)}
            if kw.get("projection") == "sign":
                # projection and tree levels, against the Gaussian build's
                comps[name]["global_ms"] = pst.ms_global
                comps[name]["global_ms_gaussian"] = st.ms_global
        eq = [v for k, v in comps.items() if k.startswith("fp32") and v["recall@10"] >= rec - 0.01]
        comps["mixed_over_plain_fp32_at_equal_recall"] = \
            min(v["ms"] for v in eq) / ms if eq else None
        mma_ms = st.ms_leaf_mma / T
        flops = 2.0 * d * st.sum_leaf_sq / T
        fp8 = prec == "fp8"
        peak = peaks.get("bf16_tflops", 1590.0) * (2 if fp8 else 1)
        roof = {"kernel": f"k_leaf_mma ({'E4M3' if fp8 else 'BF16'} tcgen05 Gram tiles + top-k "
                          "epilogue), per launch",
                "bound": "tensor", "achieved": flops / (mma_ms * 1e-3) / 1e12, "peak": peak,
                "unit": "TFLOP/s", "frac": flops / (mma_ms * 1e-3) / 1e12 / peak, "traffic": None,
                "peak_source": ("2 x " if fp8 else "") + "MEASURED_PEAKS.json bf16_tflops, the "
                               "burst figure (of measured" + ("; FP8 dense rate is twice BF16's)"
                                                              if fp8 else ")"),
                "algorithmic_flops_per_launch": flops, "ms_per_launch": mma_ms}
    cfg["comparisons"] = comps
    line = {
        "metric": METRIC, "value": n / (ms / 1e3), "unit": "points/s", "n_gpus": 1,
        "steps": steps, "warmup": warm, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": ("e4m3" if wl == "fbin-2m-960" else "bf16") + " tiles, f32 re-rank",
        "data": "synthetic", "config": cfg, "roofline": roof, "cpu_baseline": None,
        "clocks": clk, "e2e": None, "gpu_launches": launches,
    }
    print(json.dumps(line), flush=True)

# ---------------------------------------------------------------- our arm
def _traffic_per_launch(kernel: str):
    """DRAM bytes per launch of `kernel` from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        data = json.load(open(path))
        return data.get(kernel, {}).get("dram_bytes_per_launch")
    except (OSError, ValueError):
        return None


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--mode", default="mixed", choices=["mixed", "exact", "fast"])
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-plain-compare", action="store_true")
    ap.add_argument("--points", type=int, default=0,
                    help="profiling cases only: this many points of the main workload's "
                         "distribution (clusters scaled alike) instead of 1,000,000")
    ap.add_argument("--workload", default="fbin-1m-128",
                    choices=["fbin-1m-128", "ubyte-60k-784", "fbin-2m-960", "batch-256x96",
                             "learned-1m-256"])
    args = ap.parse_args()
    if args.impl == "reference":
        reference_arm(args)
        return
    if args.workload != "fbin-1m-128":
        other_workload(args)
        return
    global N_POINTS, N_CLUSTERS, WORKLOAD
    if args.points:
        # a smaller case of the same distribution, for profiling only
        N_CLUSTERS = max(1, round(N_CLUSTERS * args.points / N_POINTS))
        N_POINTS = args.points
        WORKLOAD = WORKLOAD.replace("1,000,000", f"{N_POINTS:,}").replace(
            "1000 Gaussian", f"{N_CLUSTERS} Gaussian") + " (profiling case)"

    import torch
    import torch.distributed as dist

    from drpt_b200 import build_graph, recall, synth

    world = _env_int("WORLD_SIZE", 1)
    rank = _env_int("RANK", 0)
    local_rank = _env_int("LOCAL_RANK", 0)
    if world > 1:
        from datetime import timedelta
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)

    X = synth.clustered_f32(N_POINTS, DIM, n_clusters=N_CLUSTERS, seed=2 + rank)
    Xd = torch.from_numpy(X).to(dev)
    idx = torch.empty((N_POINTS, NN), dtype=torch.int32, device=dev)
    dst = torch.empty((N_POINTS, NN), dtype=torch.float32, device=dev)
    trees = MIXED_TREES if args.mode == "mixed" else NTREES
    leaf = MIXED_LEAF if args.mode == "mixed" else 0

    def step(mode=args.mode, ntrees=trees, leaf_size=leaf, data=Xd, out=(idx, dst)):
        return build_graph(data, ntrees, NN, SEED_PROJ + rank, mode=mode, leaf_size=leaf_size,
                           out=out)[2]

    def barrier():
        if world > 1:
            dist.barrier()

    for _ in range(max(args.warmup, 3)):
        st = step()
    torch.cuda.synchronize()

    # device-resident timing
    phases = {k: [] for k in ("project", "global", "local", "leaf_knn", "merge", "leaf_mma",
                              "leaf_stage")}
    launches = 0
    with ClockSampler(local_rank) as clocks:
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            st = step()
            for k in phases:
                phases[k].append(getattr(st, "ms_" + k))
            launches += st.kernels_launched
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
    ms = e0.elapsed_time(e1) / args.steps
    if world > 1:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    clk = clocks.summary()

    # recall@10 on a seeded sample against FP64 exact neighbours
    q = recall.sample_queries(N_POINTS, 1000, seed=7)
    true_i, _ = recall.exact_knn_fp64(Xd, q, NN, device=local_rank)
    rec = recall.recall_at_k(idx.cpu().numpy()[q], true_i)

    # end to end from pinned host memory, every step copying its 512 MB of
    # rows to the device and its lists back: the pipelined call
    # (drpt_build_graph_stream: step j's input copy and step j - 1's output
    # copy overlap step j's build) over K steps, timed by the wall clock
    # around it; beside it the single host-pointer call, one step at a time
    e2e = None
    if not args.no_e2e:
        from drpt_b200 import build_graph_stream
        Xh = torch.from_numpy(X).pin_memory()
        xnp = Xh.numpy()
        bufs = [(torch.empty((N_POINTS, NN), dtype=torch.int32).pin_memory().numpy(),
                 torch.empty((N_POINTS, NN), dtype=torch.float32).pin_memory().numpy())
                for _ in range(2)]

        def stream_steps(k):
            build_graph_stream([xnp] * k, trees, NN, SEED_PROJ + rank, leaf_size=leaf,
                               outs=[bufs[j % 2] for j in range(k)], stream=stream.cuda_stream)

        def host_step():
            build_graph(xnp, trees, NN, SEED_PROJ + rank, mode=args.mode, leaf_size=leaf,
                        out=bufs[0], stream=stream.cuda_stream)

        def wall_ms(fn, k):
            barrier()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            fn()
            torch.cuda.synchronize()
            v = (time.perf_counter() - t0) * 1e3 / k
            if world > 1:
                t = torch.tensor([v], device=dev)
                dist.all_reduce(t, op=dist.ReduceOp.MAX)
                v = float(t.item())
            return v

        host_step()
        single_ms = wall_ms(lambda: [host_step() for _ in range(args.steps)], args.steps)
        e2e_ms = single_ms
        via = "drpt_build_graph (one call per step)"
        if args.mode == "mixed":
            stream_steps(max(args.warmup, 3))
            e2e_ms = wall_ms(lambda: stream_steps(args.steps), args.steps)
            via = ("drpt_build_graph_stream (K steps in one call; step j's input copy and "
                   "step j-1's output copy overlap step j's build)")
            assert np.array_equal(bufs[(args.steps - 1) % 2][0], idx.cpu().numpy()), \
                "the pipelined call's lists differ from the device-resident build's"
        e2e = {"value": world * N_POINTS / (e2e_ms / 1e3), "unit": "points/s",
               "ms_per_step": e2e_ms, "h2d_bytes_per_step": int(X.nbytes),
               "d2h_bytes_per_step": int(N_POINTS * NN * 8), "via": via,
               "single_call": {"value": world * N_POINTS / (single_ms / 1e3),
                               "ms_per_step": single_ms}}

    # the plain FP32 form beside it (one GPU only): reference parameters, and
    # grown towards the mixed form's recall, and the FP32 counterpart of the
    # mixed form (same trees, exact FP32 leaf brute force)
    plain = None
    if not args.no_plain_compare and world == 1 and args.mode == "mixed":
        plain = {}
        for name, mode, ntrees, lsz in (
                ("exact_16_trees", "exact", NTREES, 0),
                ("fast_16_trees", "fast", NTREES, 0),
                (f"fast_{PLAIN_MATCH_TREES}_trees", "fast", PLAIN_MATCH_TREES, 0),
                (f"fp32_leaf_{MIXED_TREES}_trees", "fp32_leaf", MIXED_TREES, MIXED_LEAF),
                (f"fp32_gram_{MIXED_TREES}_trees", "fp32_gram", MIXED_TREES, MIXED_LEAF)):
            pi = torch.empty((N_POINTS, NN), dtype=torch.int32, device=dev)
            pd = torch.empty((N_POINTS, NN), dtype=torch.float32, device=dev)
            step(mode, ntrees, lsz, Xd, (pi, pd))
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            pst = step(mode, ntrees, lsz, Xd, (pi, pd))
            b.record(stream)
            torch.cuda.synchronize()
            pms = a.elapsed_time(b)
            plain[name] = {"points_per_s": N_POINTS / (pms / 1e3), "ms": pms, "ntrees": ntrees,
                           "recall@10": recall.recall_at_k(pi.cpu().numpy()[q], true_i)}
            if mode == "fp32_gram":
                # its leaf phase (FFMA Gram tiles + folds): FP32 work 2 d per
                # leaf pair against the FP32 FFMA rate of 148 SMs x 128 lanes
                # x 2 flops at the sampled SM clock (MEASURED_PEAKS.json has
                # no FP32 figure)
                fl = 2.0 * DIM * pst.sum_leaf_sq
                tf = fl / (pst.ms_leaf_mma * 1e-3) / 1e12
                fp32_peak = 148 * 128 * 2 * (clk.get("sm_mhz") or 1965.0) * 1e6 / 1e12
                plain[name].update({"leaf_ms": pst.ms_leaf_mma, "leaf_tflops": tf,
                                    "leaf_frac_of_fp32_ffma_peak": tf / fp32_peak})
            del pi, pd
        # Equal recall: only the FP32 whole-leaf forms (same trees and leaves
        # as the mixed form: exact per-pair distances, or FFMA Gram tiles with
        # an FP32 re-rank) reach it; the reference's positional local split
        # saturates far below (see fast_{PLAIN_MATCH_TREES}_trees).  The ratio
        # is taken against the fastest of them.
        eq = [v for v in plain.values() if v["recall@10"] >= rec - 0.01]
        best_plain = max(v["points_per_s"] for v in eq) if eq else None
        plain["mixed_over_plain_fp32_at_equal_recall"] = \
            (world * N_POINTS / (ms / 1e3)) / best_plain if best_plain else None

    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return

    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    if args.mode == "mixed":
        # dominant kernel: the tensor-core leaf kernel (one launch per tree);
        # algorithmic work = 2*d multiply-adds per leaf pair
        mma_ms = statistics.median(phases["leaf_mma"]) / trees
        flops = 2.0 * DIM * st.sum_leaf_sq / trees
        achieved = flops / (mma_ms * 1e-3) / 1e12
        # one launch lasts about a millisecond: the burst figure is its peak
        peak = peaks.get("bf16_tflops", 1590.0)
        roofline = {"kernel": "k_leaf_mma (BF16 tcgen05 Gram tiles + top-k epilogue) and, from "
                              "the second tree, k_fold_lists: the leaf phase of one tree",
                    "bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                    "frac": achieved / peak, "traffic": _traffic_per_launch("k_leaf_mma"),
                    "traffic_source": "profiles/traffic.json: DRAM bytes per launch from an ncu "
                                      "capture of this kernel (not measured in this run)",
                    "peak_source": ("MEASURED_PEAKS.json bf16_tflops, the burst figure (of measured)"
                                    if "bf16_tflops" in peaks else "fallback 1590 TFLOP/s (of fallback)"),
                    "algorithmic_flops_per_launch": flops, "ms_per_launch": mma_ms,
                    "padded_tile_flops_per_launch": 2.0 * 128 * st.mma_pairs_padded / trees,
                    "note": "the epilogue (threshold filter + bitonic top-k in registers) bounds "
                            "this kernel, not the tensor pipe"}
    else:
        leaf_ms = statistics.median(phases["leaf_knn"])
        flops = 3.0 * st.sum_leaf_sq * DIM
        achieved = flops / (leaf_ms * 1e-3) / 1e12
        sm_mhz = clk.get("sm_mhz") or peaks.get("sm_max_mhz", 1965.0)
        fp32_peak = 148 * 128 * sm_mhz * 1e6 / 1e12
        roofline = {"kernel": "k_leaf_knn (exact FP32 leaf brute force)", "bound": "fp32",
                    "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                    "frac": achieved / fp32_peak, "traffic": _traffic_per_launch("k_leaf_knn"),
                    "peak_source": "nominal FP32 issue rate (148 SMs x 128 lanes x median SM "
                                   "clock); MEASURED_PEAKS.json holds no FP32 figure",
                    "algorithmic_flops_per_launch": flops}
    cpu = None
    if not args.no_cpu_baseline and world == 1:
        try:
            cpu = cpu_baseline()
        except Exception as ex:  # reported, not fatal
            cpu = {"value": None, "unit": "points/s", "error": str(ex)[:200]}
    line = {
        "metric": METRIC, "value": world * N_POINTS / (ms / 1e3), "unit": "points/s",
        "n_gpus": world, "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "bf16 tiles, f32 re-rank" if args.mode == "mixed" else "f32",
        "data": "synthetic",
        "config": {"workload": WORKLOAD,
                   "trees": TREES_MIXED if args.mode == "mixed" else TREES_REFERENCE,
                   "mode": args.mode, "ntrees": trees,
                   "leaf_size": leaf or None, "recall@10": rec, "recall_sample": 1000,
                   "global_depth": st.global_depth, "local_depth": st.local_depth,
                   "mean_leaf": st.sum_leaf_sq / (trees * N_POINTS),
                   "phase_ms": {k: statistics.median(v) for k, v in phases.items()},
                   "plain_form": plain,
                   "l2": "input 512 MB > 126 MB L2; no flush between steps",
                   "parallelism": f"replicas x{world}" if world > 1 else "1 GPU"},
        "roofline": roofline, "cpu_baseline": cpu, "clocks": clk, "e2e": e2e,
        "gpu_launches": launches,
    }
    if rank == 0:  # one line per job; every rank's timing is already max-reduced
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
