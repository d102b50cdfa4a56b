"""drpt_global_trees_noalloc, the global-tree build for callers that cannot
allocate device memory (hosts whose own pool holds the GPU's memory, loops
that cannot take cudaMalloc's synchronisation).  It keeps its scratch in a
fixed array inside the library instead of a cudaMalloc'd workspace, so its
outputs must equal drpt_global_trees's on the same inputs.  Tree order,
leaf offsets and medians are integer or bit-exact results: the tolerance is
zero.

The file sorts last so that a run stopping at the first failure has run
every other test before it; it also passes alone in a fresh process."""
import ctypes

import numpy as np
import pytest

from drpt_b200 import _lib

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as _t
    if not _t.cuda.is_available():
        pytest.skip("no CUDA device")
    return _t


def _projected(torch, n, T, gd, seed):
    """(T*(gd-1)) x n projected columns: clustered values with exact ties,
    so that medians, empty histogram slots and equal keys all occur."""
    rng = np.random.default_rng(seed)
    cols = max(T * (gd - 1), 1)
    centres = rng.uniform(-50, 50, size=(cols, 64)).astype(np.float32)
    pick = rng.integers(0, 64, size=n)
    P = centres[:, pick] + rng.standard_normal((cols, n)).astype(np.float32)
    P[:, ::97] = np.round(P[:, ::97])
    return torch.from_numpy(np.ascontiguousarray(P)).cuda()


def _outputs(torch, n, T, gd):
    nleaf = 1 << (gd - 1)
    order = torch.full((T, n), -7, dtype=torch.int32, device="cuda")
    offs = torch.full((T, nleaf + 1), -7, dtype=torch.int32, device="cuda")
    med = torch.full((T, max(nleaf - 1, 1)), float("nan"), dtype=torch.float32, device="cuda")
    return order, offs, med


def _with_workspace(torch, P, n, T, gd, exact):
    L = _lib.load()
    ctx = _lib.context(0)
    order, offs, med = _outputs(torch, n, T, gd)
    s = torch.cuda.current_stream().cuda_stream
    _lib.check(L.drpt_global_trees(ctx.handle, P.data_ptr(), n, T, gd, exact, order.data_ptr(),
                                   offs.data_ptr(), med.data_ptr(), s))
    torch.cuda.synchronize()
    return order.cpu().numpy(), offs.cpu().numpy(), med.cpu().numpy()


def _without_alloc(torch, P, n, T, gd, exact):
    L = _lib.load()
    order, offs, med = _outputs(torch, n, T, gd)
    s = torch.cuda.current_stream().cuda_stream
    _lib.check(L.drpt_global_trees_noalloc(P.data_ptr(), n, T, gd, exact, order.data_ptr(),
                                           offs.data_ptr(), med.data_ptr(), s))
    torch.cuda.synchronize()
    return order.cpu().numpy(), offs.cpu().numpy(), med.cpu().numpy()


def test_noalloc_equals_workspace_entry_on_calls_in_a_row(torch):
    # Consecutive calls of different shapes: each one starts with the previous
    # call's contents in the shared static scratch.
    # Odd and even global depths: with even gd the last level ends in the
    # other side of the ping-pong, and at gd = 2 the ping-pong side, the
    # split values and the offsets side are not carved at all.
    for n, T, gd, exact in [(200_000, 4, 7, 1), (150_001, 6, 5, 0), (200_000, 4, 7, 1),
                            (100_000, 4, 2, 1), (150_001, 6, 6, 1), (120_000, 5, 4, 0),
                            (90_001, 3, 2, 0), (1_000, 3, 1, 1)]:
        P = _projected(torch, n, T, gd, seed=n + T + gd)
        want = _with_workspace(torch, P, n, T, gd, exact)
        got = _without_alloc(torch, P, n, T, gd, exact)
        nleaf = 1 << (gd - 1)
        assert np.array_equal(got[0], want[0]), (n, T, gd, exact)
        assert np.array_equal(got[1], want[1]), (n, T, gd, exact)
        if gd > 1:
            assert got[2][:, :nleaf - 1].tobytes() == want[2][:, :nleaf - 1].tobytes()
        assert (got[1][:, -1] == n).all() and (got[1][:, 0] == 0).all()


def test_noalloc_rejects_builds_beyond_its_scratch(torch):
    # 2M points x 16 trees needs ~400 MB of scratch, beyond the 64 MiB array;
    # the size check runs before any launch, so the small P is never read.
    P = torch.zeros((16, 16), dtype=torch.float32, device="cuda")
    order = torch.zeros((1, 1), dtype=torch.int32, device="cuda")
    L = _lib.load()
    st = L.drpt_global_trees_noalloc(P.data_ptr(), 2_000_000, 16, 10, 1, order.data_ptr(),
                                     order.data_ptr(), None, ctypes.c_void_p(0))
    assert st == 1  # DRPT_ERR_INVALID_ARG
    msg = L.drpt_last_error().decode()
    assert "static scratch" in msg and "bytes" in msg


def test_noalloc_argument_checks_set_the_error_text(torch):
    # Every rejected argument returns DRPT_ERR_INVALID_ARG before any launch
    # and leaves a message of its own, not the text of an earlier failure.
    L = _lib.load()
    P = torch.zeros((8, 64), dtype=torch.float32, device="cuda")
    order = torch.zeros((1, 64), dtype=torch.int32, device="cuda")
    offs = torch.zeros((1, 64), dtype=torch.int32, device="cuda")
    s = ctypes.c_void_p(0)
    cases = [
        ((None, 64, 1, 3, 1, order.data_ptr(), offs.data_ptr(), None, s), "device pointers"),
        ((P.data_ptr(), 64, 1, 3, 1, None, offs.data_ptr(), None, s), "device pointers"),
        ((P.data_ptr(), 64, 1, 3, 1, order.data_ptr(), None, None, s), "device pointers"),
        ((P.data_ptr(), 1, 1, 3, 1, order.data_ptr(), offs.data_ptr(), None, s), "out of range"),
        ((P.data_ptr(), 64, 0, 3, 1, order.data_ptr(), offs.data_ptr(), None, s), "out of range"),
        ((P.data_ptr(), 64, 1, 0, 1, order.data_ptr(), offs.data_ptr(), None, s), "out of range"),
        ((P.data_ptr(), 64, 1, 31, 1, order.data_ptr(), offs.data_ptr(), None, s), "out of range"),
    ]
    for args, words in cases:
        # plant an unrelated message first: the check must replace it
        assert L.drpt_global_trees_noalloc(P.data_ptr(), 2_000_000, 16, 10, 1, order.data_ptr(),
                                           offs.data_ptr(), None, s) == 1
        assert "static scratch" in L.drpt_last_error().decode()
        assert L.drpt_global_trees_noalloc(*args) == 1, args
        msg = L.drpt_last_error().decode()
        assert words in msg and "static scratch" not in msg, (args, msg)
