"""A small, self-contained build for profiling one kernel under ncu.

    python -m drpt_b200.profile_case --n 262144 --dim 128 --trees 4 --mode exact --reps 2
    python -m drpt_b200.profile_case --n 200000 --dim 960 --data anisotropic --nn 20 \\
        --trees 2 --mode mixed --leaf 2048 --precision fp8
    python -m drpt_b200.profile_case --n 200000 --dim 256 --data manifold --trees 4 \\
        --learned 4 --mode mixed --leaf 1024

Data: `clustered` (the benchmark workload's distribution: Gaussian clusters,
centres U[0,200]^d, sigma 12, clipped to [0,255]), `anisotropic` (per-dim
sigma U[0.01,0.3] in [0,1]) or `manifold` (16-dim latent manifold); fewer
points and trees than the benchmarks so that a capture of one or two
launches ends within a minute.
"""
from __future__ import annotations

import argparse

import torch

from drpt_b200 import build_graph, synth


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=262_144)
    ap.add_argument("--dim", type=int, default=128)
    ap.add_argument("--trees", type=int, default=4)
    ap.add_argument("--nn", type=int, default=10)
    ap.add_argument("--mode", default="exact")
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--leaf", type=int, default=0, help="mixed mode: target leaf size")
    ap.add_argument("--precision", default="bf16", choices=["bf16", "fp8"])
    ap.add_argument("--learned", type=int, default=0, help="mixed mode: learned trees")
    ap.add_argument("--learn-sample", type=int, default=0, help="learned trees: sample size")
    ap.add_argument("--data", default="clustered", choices=["clustered", "anisotropic", "manifold"])
    args = ap.parse_args()
    if args.data == "clustered":
        X = synth.clustered_f32(args.n, args.dim, n_clusters=max(1, args.n // 1000), seed=2)
    elif args.data == "anisotropic":
        X = synth.anisotropic_f32(args.n, args.dim, n_clusters=max(1, args.n // 4000), seed=3)
    else:
        X = synth.latent_manifold_f32(args.n, args.dim, seed=5)
    Xd = torch.from_numpy(X).cuda()
    for _ in range(args.reps):
        _, _, st = build_graph(Xd, args.trees, args.nn, 12345, mode=args.mode, leaf_size=args.leaf,
                               precision=args.precision, learned_trees=args.learned,
                               learn_sample=args.learn_sample)
    torch.cuda.synchronize()
    print({k: round(v, 3) if isinstance(v, float) else v for k, v in st.as_dict().items()})


if __name__ == "__main__":
    main()
