"""The sign-matrix projection of u8 rows on the tensor cores (K1u,
tcgen05.mma kind::i8): exact against the integer product on the CPU, and as
the projection of the mixed form, judged by recall against FP64 exact
neighbours next to the reference's Gaussian projection."""
import ctypes

import numpy as np
import pytest

from drpt_b200 import DrptError, _lib, build_graph, recall, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as _t
    if not _t.cuda.is_available():
        pytest.skip("no CUDA device")
    return _t


def _sign_project(torch, X, B, cols):
    L = _lib.load()
    ctx = _lib.context(0)
    n, d = X.shape
    Xd = torch.from_numpy(X).cuda()
    P = torch.full((len(cols), n), float("nan"), dtype=torch.float32, device="cuda")
    c = np.ascontiguousarray(cols, np.int32)
    Bc = np.ascontiguousarray(B, np.float32)
    _lib.check(L.drpt_project_sign(ctx.handle, Xd.data_ptr(), n, d, Bc.ctypes.data,
                                   B.shape[1], c.ctypes.data, len(cols), P.data_ptr(),
                                   torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return P.cpu().numpy()


@pytest.mark.parametrize("n,d,L,ncols", [(10_001, 784, 320, 300), (777, 128, 40, 37),
                                         (4_096, 96, 16, 16)])
def test_sign_projection_is_the_exact_integer_product(torch, n, d, L, ncols):
    rng = np.random.default_rng(n + d)
    X = rng.integers(0, 256, size=(n, d)).astype(np.uint8)
    X[::7] = 255  # the largest sums: 255 * (non-zeros of a column)
    B = np.empty((d, L), np.float32)
    _lib.check(_lib.load().drpt_host_projection(4321, d, L, ctypes.c_float(1.0 / np.sqrt(d)),
                                                B.ctypes.data))
    cols = rng.permutation(L)[:ncols]
    got = _sign_project(torch, X, B, cols)
    S = np.sign(B[:, cols]).astype(np.int64)
    want = (X.astype(np.int64) @ S).T.astype(np.float32)
    assert np.array_equal(got, want)


def test_mixed_form_with_the_sign_projection(torch):
    X = synth.clustered_u8(60_000, 784, seed=1)
    Xd = torch.from_numpy(X).cuda()
    q = recall.sample_queries(len(X), 400, seed=5)
    ti, _ = recall.exact_knn_fp64(Xd, q, 10)
    gi, _, _ = build_graph(Xd, 12, 10, 12345, mode="mixed", leaf_size=1024)
    si, sd, st = build_graph(Xd, 12, 10, 12345, mode="mixed", leaf_size=1024, projection="sign")
    torch.cuda.synchronize()
    rg = recall.recall_at_k(gi.cpu().numpy()[q], ti)
    rs = recall.recall_at_k(si.cpu().numpy()[q], ti)
    assert rs >= rg - 0.03 and rs >= 0.9, (rs, rg)
    # deterministic
    s2, _, _ = build_graph(Xd, 12, 10, 12345, mode="mixed", leaf_size=1024, projection="sign")
    torch.cuda.synchronize()
    assert torch.equal(si, s2)


def test_sign_projection_limits(torch):
    Xf = synth.clustered_f32(5_000, 64, n_clusters=10, seed=2)
    with pytest.raises(DrptError):
        build_graph(Xf, 4, 10, 1, mode="mixed", projection="sign")  # f32 rows
    Xu = synth.clustered_u8(5_000, 100, sigma_p=40.0, seed=2)
    with pytest.raises(DrptError):
        build_graph(Xu, 4, 10, 1, mode="mixed", projection="sign")  # d % 16 != 0
    with pytest.raises(DrptError):
        build_graph(Xu, 4, 10, 1, mode="exact", projection="sign")  # not the exact form
