"""Seeded synthetic inputs with the shapes and value distributions of the five
k-NN-graph workloads (the reference's MNIST file is not available, and none of
its items is reproduced here), plus writers for the two input formats the
`drpt` command line reads.

Formats (reference readers: cpp/src/drpt/io/file_reader.cpp):
  * ubyte / IDX3 (read_ubyte, file_reader.cpp:33-87): big-endian header
    0x00000803, N, rows, cols, then N*rows*cols bytes, uncompressed.
  * fbin (mpi_file_read, file_reader.cpp:364-493 with -data-starting-index 8):
    u32 N, u32 d, then N*d little-endian float32.
"""
from __future__ import annotations

import struct

import numpy as np

__all__ = [
    "clustered_u8", "clustered_f32", "anisotropic_f32", "batch_sizes", "batch_dataset",
    "latent_manifold_f32", "write_idx3", "write_fbin", "read_idx3", "read_fbin",
]


def clustered_u8(n: int = 60_000, d: int = 784, n_centres: int = 10, zero_frac: float = 0.8,
                 sigma_p: float = 20.0, seed: int = 1) -> np.ndarray:
    """MNIST-shaped u8 data: `n_centres` centres, each with `zero_frac` of its
    coordinates forced to 0 and the rest N(128, 60^2) clipped to [0, 255]; a
    point picks a centre uniformly, keeps its zero support and draws
    round(centre + N(0, sigma_p^2)) clipped to [0, 255] elsewhere."""
    rng = np.random.default_rng(seed)
    centres = np.clip(rng.normal(128.0, 60.0, size=(n_centres, d)), 0, 255)
    support = rng.random((n_centres, d)) >= zero_frac
    centres = centres * support
    which = rng.integers(0, n_centres, size=n)
    out = np.empty((n, d), dtype=np.uint8)
    chunk = 8192
    for s in range(0, n, chunk):
        w = which[s:s + chunk]
        x = centres[w] + rng.normal(0.0, sigma_p, size=(len(w), d))
        x = np.clip(np.rint(x), 0, 255) * support[w]
        out[s:s + chunk] = x.astype(np.uint8)
    return out


def clustered_f32(n: int = 1_000_000, d: int = 128, n_clusters: int = 1000, lo: float = 0.0,
                  hi: float = 200.0, sigma: float = 12.0, clip=(0.0, 255.0),
                  seed: int = 2) -> np.ndarray:
    """Isotropic Gaussian mixture: centres U[lo, hi]^d, per-point noise
    N(0, sigma^2), values clipped to `clip`, float32."""
    rng = np.random.default_rng(seed)
    centres = rng.uniform(lo, hi, size=(n_clusters, d)).astype(np.float32)
    which = rng.integers(0, n_clusters, size=n)
    out = np.empty((n, d), dtype=np.float32)
    chunk = 65536
    for s in range(0, n, chunk):
        w = which[s:s + chunk]
        x = centres[w] + rng.standard_normal(size=(len(w), d), dtype=np.float32) * np.float32(sigma)
        if clip is not None:
            np.clip(x, clip[0], clip[1], out=x)
        out[s:s + chunk] = x
    return out


def anisotropic_f32(n: int = 2_000_000, d: int = 960, n_clusters: int = 500,
                    seed: int = 3) -> np.ndarray:
    """Anisotropic mixture: centres U[0,1]^d, per-cluster per-dim sigma
    U[0.01, 0.3], values clipped to [0, 1]."""
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0.0, 1.0, size=(n_clusters, d)).astype(np.float32)
    sig = rng.uniform(0.01, 0.3, size=(n_clusters, d)).astype(np.float32)
    which = rng.integers(0, n_clusters, size=n)
    out = np.empty((n, d), dtype=np.float32)
    chunk = 16384
    for s in range(0, n, chunk):
        w = which[s:s + chunk]
        x = centres[w] + rng.standard_normal(size=(len(w), d), dtype=np.float32) * sig[w]
        np.clip(x, 0.0, 1.0, out=x)
        out[s:s + chunk] = x
    return out


def batch_sizes(count: int = 256, lo: int = 2_000, hi: int = 200_000, seed: int = 4) -> np.ndarray:
    """Dataset sizes log-uniform in [lo, hi]."""
    rng = np.random.default_rng(seed)
    return np.exp(rng.uniform(np.log(lo), np.log(hi), size=count)).astype(np.int64)


def batch_dataset(n: int, d: int = 96, seed: int = 0) -> np.ndarray:
    """One dataset of the batched workload: 20-200 Gaussians, sigma 1,
    centres U[-10, 10]^d, float32."""
    rng = np.random.default_rng(seed)
    k = int(rng.integers(20, 201))
    centres = rng.uniform(-10.0, 10.0, size=(k, d)).astype(np.float32)
    which = rng.integers(0, k, size=n)
    return (centres[which] + rng.standard_normal(size=(n, d), dtype=np.float32)).astype(np.float32)


def latent_manifold_f32(n: int = 1_000_000, d: int = 256, latent: int = 16, seed: int = 5) -> np.ndarray:
    """x = tanh(A z + b) * 4 + N(0, 0.05^2) with z ~ N(0, I_latent),
    A (d x latent) and b seeded Gaussians."""
    rng = np.random.default_rng(seed)
    A = rng.standard_normal(size=(d, latent)).astype(np.float32)
    b = rng.standard_normal(size=(d,)).astype(np.float32)
    out = np.empty((n, d), dtype=np.float32)
    chunk = 65536
    for s in range(0, n, chunk):
        m = min(chunk, n - s)
        z = rng.standard_normal(size=(m, latent), dtype=np.float32)
        x = np.tanh(z @ A.T + b) * np.float32(4.0)
        x += rng.standard_normal(size=(m, d), dtype=np.float32) * np.float32(0.05)
        out[s:s + m] = x
    return out


def write_idx3(path: str, x: np.ndarray, rows: int | None = None, cols: int | None = None) -> None:
    """Uncompressed IDX3: big-endian magic 0x00000803, N, rows, cols; u8 data."""
    x = np.ascontiguousarray(x, dtype=np.uint8)
    n, d = x.shape
    if rows is None:
        rows = int(round(d ** 0.5))
        cols = d // rows
    assert rows * cols == d, "IDX3 needs rows*cols == d"
    with open(path, "wb") as f:
        f.write(struct.pack(">iiii", 0x00000803, n, rows, cols))
        f.write(x.tobytes())


def write_fbin(path: str, x: np.ndarray) -> None:
    """fbin: little-endian u32 N, u32 d, then N*d float32."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    n, d = x.shape
    with open(path, "wb") as f:
        f.write(struct.pack("<II", n, d))
        f.write(x.tobytes())


def read_idx3(path: str) -> np.ndarray:
    with open(path, "rb") as f:
        magic, n, r, c = struct.unpack(">iiii", f.read(16))
        return np.frombuffer(f.read(n * r * c), dtype=np.uint8).reshape(n, r * c)


def read_fbin(path: str) -> np.ndarray:
    with open(path, "rb") as f:
        n, d = struct.unpack("<II", f.read(8))
        return np.frombuffer(f.read(n * d * 4), dtype=np.float32).reshape(n, d)
