"""The command line's readers under AddressSanitizer and UBSan: the CLI is
rebuilt with the sanitizers (against the same library) and given truncated,
mislabelled and corrupt inputs; each ends with status 1 before any GPU work
and without a sanitizer report.  No GPU needed."""
import gzip
import os
import shutil
import struct
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "drpt_b200")


@pytest.mark.skipif(shutil.which("g++") is None or
                    not os.path.exists(os.path.join(PKG, "libdrpt_gpu.so")),
                    reason="needs g++ and the built library")
def test_cli_readers_under_sanitizers(tmp_path):
    exe = tmp_path / "drpt_asan"
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-g", "-fno-omit-frame-pointer",
                        "-fsanitize=address,undefined", "-I", os.path.join(ROOT, "include"),
                        os.path.join(PKG, "csrc", "cli", "drpt_main.cpp"), "-o", str(exe),
                        "-L" + PKG, "-ldrpt_gpu", "-Wl,-rpath," + PKG, "-lz"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    p = lambda name: str(tmp_path / name)  # noqa: E731
    open(p("short.fbin"), "wb").write(struct.pack("<II", 1000, 16) + b"\0" * 100)
    open(p("badhdr.fbin"), "wb").write(struct.pack("<II", 999, 16) +
                                       np.zeros((1000, 16), np.float32).tobytes())
    open(p("badmagic.idx3"), "wb").write(struct.pack(">IIII", 0x801, 1000, 28, 28) + b"\0" * 784000)
    open(p("short.idx3"), "wb").write(struct.pack(">IIII", 0x803, 1000, 28, 28) + b"\0" * 1000)
    open(p("garbage.gz"), "wb").write(b"\x1f\x8b" + np.random.default_rng(1).bytes(500))
    with gzip.open(p("trunc.fbin.gz"), "wb") as f:
        f.write(struct.pack("<II", 1000, 16) + b"\1" * 2000)
    cases = [("short.fbin", 1, 16), ("badhdr.fbin", 1, 16), ("badmagic.idx3", 0, 784),
             ("short.idx3", 0, 784), ("garbage.gz", 1, 16), ("trunc.fbin.gz", 1, 16),
             ("missing.fbin", 1, 16)]
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:protect_shadow_gap=0",
               UBSAN_OPTIONS="print_stacktrace=1")
    os.makedirs(p("out"))
    for name, fmt, d in cases:
        args = [str(exe), "-input", p(name), "-output", p("out") + "/", "-data-set-size", "1000",
                "-dimension", str(d), "-ntrees", "4", "-nn", "10", "-data-file-format", str(fmt)]
        if fmt == 1:
            args += ["-bytes-for-data-type", "4", "-data-starting-index", "8"]
        r = subprocess.run(args, capture_output=True, text=True, env=env, timeout=120)
        assert r.returncode == 1, (name, r.returncode, r.stdout[-500:], r.stderr[-500:])
        for mark in ("AddressSanitizer", "LeakSanitizer", "runtime error"):
            assert mark not in r.stderr, (name, r.stderr[-3000:])
