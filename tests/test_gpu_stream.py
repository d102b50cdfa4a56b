"""The pipelined many-builds call (drpt_build_graph_stream) through the C ABI:
every job's graph equals the single host-pointer build of the same dataset,
bit for bit, with the copies of neighbouring jobs overlapping its build."""
import numpy as np
import pytest

from drpt_b200 import DrptError, build_graph, build_graph_stream, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as _t
    if not _t.cuda.is_available():
        pytest.skip("no CUDA device")
    return _t


def test_stream_jobs_equal_single_builds(torch):
    sets = [synth.clustered_f32(20_000, 64, n_clusters=40, seed=s) for s in (31, 32, 33)]
    pinned = [torch.from_numpy(x).pin_memory().numpy() for x in sets]
    outs, st = build_graph_stream(pinned, 4, 10, 777, leaf_size=512)
    assert st.ms_total > 0 and st.kernels_launched > 0
    for x, (i2, d2) in zip(sets, outs):
        i1, d1, _ = build_graph(x, 4, 10, 777, mode="mixed", leaf_size=512)
        assert np.array_equal(i1, i2)
        assert d1.tobytes() == d2.tobytes()


def test_stream_one_job_and_u8(torch):
    x = synth.clustered_u8(6_000, 784, sigma_p=40.0, seed=3)
    outs, _ = build_graph_stream([x], 3, 10, 5, leaf_size=512)
    i1, d1, _ = build_graph(x, 3, 10, 5, mode="mixed", leaf_size=512)
    assert np.array_equal(i1, outs[0][0]) and d1.tobytes() == outs[0][1].tobytes()


def test_stream_rejects_mixed_shapes_and_bad_parameters(torch):
    a = synth.clustered_f32(5_000, 32, n_clusters=10, seed=1)
    b = synth.clustered_f32(4_000, 32, n_clusters=10, seed=2)
    with pytest.raises(ValueError):
        build_graph_stream([a, b], 2, 10, 1)
    with pytest.raises(DrptError) as e:
        build_graph_stream([a], 2, 40, 1)  # nn > 32 in the mixed form
    assert e.value.status_name in ("DRPT_ERR_UNSUPPORTED", "DRPT_ERR_INVALID_ARG")
