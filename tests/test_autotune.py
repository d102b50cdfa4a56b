"""The autotuner's choice rule and its cache (no GPU needed)."""
import pytest

from drpt_b200 import autotune


def test_choose_fastest_that_reaches_the_target():
    trials = [{"leaf_size": 256, "list_width": 16, "ms": 10.0, "recall": 0.88},
              {"leaf_size": 512, "list_width": 16, "ms": 14.0, "recall": 0.91},
              {"leaf_size": 512, "list_width": 32, "ms": 20.0, "recall": 0.93},
              {"leaf_size": 1024, "list_width": 16, "ms": 12.0, "recall": 0.92}]
    assert autotune.choose(trials, 0.90)["leaf_size"] == 1024
    assert autotune.choose(trials, 0.925)["list_width"] == 32
    # none reaches the target: the most accurate
    assert autotune.choose(trials, 0.99)["recall"] == 0.93


def test_widths_hold_nn():
    assert autotune._widths(10, None) == [16, 32]
    assert autotune._widths(16, None) == [16, 32]
    assert autotune._widths(20, None) == [32]
    with pytest.raises(ValueError):
        autotune._widths(40, None)


def test_cache_round_trip(tmp_path):
    path = str(tmp_path / "tune.json")
    assert autotune._load_cache(path, "k") is None
    autotune._store_cache(path, "k", {"leaf_size": 512, "list_width": 16})
    autotune._store_cache(path, "k2", {"leaf_size": 256, "list_width": 32})
    assert autotune._load_cache(path, "k") == {"leaf_size": 512, "list_width": 16}
    assert autotune._load_cache(path, "k2")["list_width"] == 32
