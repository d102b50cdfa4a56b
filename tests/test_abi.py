"""The C ABI boundary without a GPU: the library loads, exports every
function include/drpt_gpu.h declares, its host-side projection matrix is the
reference's, and calls that need a device fail with a status instead of
crashing."""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle
from drpt_b200 import _lib
from tests.conftest import GOLDEN, ROOT

HEADER = os.path.join(ROOT, "include", "drpt_gpu.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(drpt_[a-z_]+)\s*\(", text)))


def test_header_matches_binding():
    assert declared_functions() == sorted(_lib.EXPORTS)


def test_library_exports_every_declared_symbol():
    L = _lib.load()
    for name in declared_functions():
        assert hasattr(L, name), name


def test_version_and_last_error():
    L = _lib.load()
    assert L.drpt_version().decode().startswith("drpt-b200")
    assert isinstance(L.drpt_last_error(), bytes)


@pytest.mark.parametrize("case", ["u8_c1", "f32_c2", "f32_odd", "u8_ties"])
def test_host_projection_is_the_reference_matrix(case):
    g = np.load(os.path.join(GOLDEN, f"case_{case}.npz"))
    d = g["X"].shape[1]
    L = int(g["gd"]) * int(g["ntrees"])
    B = np.empty((d, L), np.float32)
    _lib.check(_lib.load().drpt_host_projection(int(g["seeds"][0]), d, L,
                                                ctypes.c_float(float(g["density"])), B.ctypes.data))
    assert np.array_equal(B, g["B"])
    assert np.array_equal(B, oracle.projection_matrix(int(g["seeds"][0]), d, L, float(g["density"])))


def test_invalid_arguments_return_status():
    L = _lib.load()
    assert L.drpt_host_projection(1, 0, 4, ctypes.c_float(0.5), None) == 1
    assert L.drpt_build_graph(None, None, None, None, None, None) == 1


def test_context_without_device_reports_error():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    h = ctypes.c_void_p()
    st = _lib.load().drpt_ctx_create(ctypes.byref(h), 0)
    assert st in (1, 6)  # invalid device or CUDA error, never a crash


def test_struct_layouts_match_the_header(tmp_path):
    """The ctypes mirrors of drpt_build_desc, drpt_stats and drpt_batch_desc
    have the C header's sizes and field offsets (compiled with the system C
    compiler)."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    checks = []
    for cname, py in (("drpt_build_desc", _lib.BuildDesc), ("drpt_stats", _lib.Stats),
                      ("drpt_batch_desc", _lib.BatchDesc)):
        checks.append((f"sizeof({cname})", ctypes.sizeof(py)))
        for field, _ in py._fields_:
            checks.append((f"offsetof({cname}, {field})", getattr(py, field).offset))
    src = tmp_path / "layout.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "drpt_gpu.h"\nint main(void) {\n' +
                   "".join(f'  printf("%zu\\n", (size_t){expr});\n' for expr, _ in checks) +
                   "  return 0;\n}\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True,
                                          check=True).stdout.split()]
    assert got == [v for _, v in checks]
