"""The library's host-side C++ (the seeded projection matrix, the positional
local split and the locality relabelling, csrc/host_algo.cpp) built on its
own with AddressSanitizer and UndefinedBehaviorSanitizer and run on golden
inputs: no sanitizer report, and the same results as the library's C ABI.
No GPU needed."""
import ctypes
import glob
import os
import shutil
import subprocess

import numpy as np
import pytest

from drpt_b200 import _lib
from tests.conftest import GOLDEN
from tests.test_locality import _global_leaves

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "drpt_b200", "csrc")

DRIVER = r"""
#include <cstdio>
#include <cstdlib>
#include <vector>
#include "host_algo.h"

static std::vector<int32_t> read_i32(const char *p, size_t n) {
  std::vector<int32_t> v(n);
  FILE *f = std::fopen(p, "rb");
  if (!f || std::fread(v.data(), 4, n, f) != n) std::exit(3);
  std::fclose(f);
  return v;
}

int main(int argc, char **argv) {
  // 1: projection matrix, written to argv[2]
  const int d = 37, L = 11;
  std::vector<float> B((size_t)d * L);
  drpt::host_projection_matrix(12345u, d, L, 0.2f, B.data());
  FILE *f = std::fopen(argv[1], "wb");
  std::fwrite(B.data(), 4, B.size(), f);
  std::fclose(f);
  // 2: positional split of several leaf sizes and depths
  for (int n : {1, 2, 3, 7, 64, 1000, 4099})
    for (int ld = 1; ld <= 5; ++ld) {
      std::vector<int32_t> perm, first;
      drpt::host_local_permutation(n, ld, perm, first);
      if ((int)perm.size() != n || first.back() != n) return 4;
    }
  // 3: locality slots of the golden global leaves in argv[2] (T, nleaf, n, order, goff)
  const std::vector<int32_t> hdr = read_i32(argv[2], 3);
  const int T = hdr[0], nleaf = hdr[1], n = hdr[2];
  std::vector<int32_t> all = read_i32(argv[2], 3 + (size_t)T * n + (size_t)T * (nleaf + 1));
  const int32_t *order = all.data() + 3, *goff = order + (size_t)T * n;
  std::vector<int32_t> slots((size_t)nleaf * T, -1);
  if (!drpt::host_locality_slots(T, nleaf, n, order, goff, slots.data())) return 5;
  f = std::fopen(argv[3], "wb");
  std::fwrite(slots.data(), 4, slots.size(), f);
  std::fclose(f);
  return 0;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_host_code_under_sanitizers(tmp_path):
    src = tmp_path / "driver.cpp"
    src.write_text(DRIVER)
    exe = tmp_path / "driver"
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-g", "-fno-omit-frame-pointer",
                        "-fsanitize=address,undefined", "-fno-sanitize-recover=all",
                        "-I", CSRC, str(src), os.path.join(CSRC, "host_algo.cpp"), "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    case = sorted(glob.glob(os.path.join(GOLDEN, "case_f32_c2.npz")))[0]
    g = np.load(case)
    nleaf = 1 << (int(g["gd"]) - 1)
    go, gf = _global_leaves(g["final_order"], g["final_offsets"], nleaf)
    T, n = go.shape
    leaves = tmp_path / "leaves.bin"
    np.concatenate([np.array([T, nleaf, n], np.int32), go.ravel(), gf.ravel()]).astype(
        np.int32).tofile(leaves)
    bpath, spath = tmp_path / "B.bin", tmp_path / "slots.bin"
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:abort_on_error=0",
               UBSAN_OPTIONS="print_stacktrace=1")
    r = subprocess.run([str(exe), str(bpath), str(leaves), str(spath)], capture_output=True,
                       text=True, env=env, timeout=300)
    assert r.returncode == 0, (r.returncode, r.stderr[-3000:])
    assert "runtime error" not in r.stderr and "AddressSanitizer" not in r.stderr
    # the same results through the library
    L = _lib.load()
    want_B = np.empty((37, 11), np.float32)
    _lib.check(L.drpt_host_projection(12345, 37, 11, ctypes.c_float(0.2), want_B.ctypes.data))
    assert np.fromfile(bpath, np.float32).tobytes() == want_B.tobytes()
    want_s = np.full((nleaf, T), -1, np.int32)
    _lib.check(L.drpt_locality_slots(go.ctypes.data, gf.ctypes.data, n, T, nleaf,
                                     want_s.ctypes.data, None, None))
    assert np.array_equal(np.fromfile(spath, np.int32).reshape(nleaf, T), want_s)
