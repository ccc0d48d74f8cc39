"""The autotuner's choice cache and the batch scheduler's station masks, on
the CPU: cache keys per GPU / storage / reduce / stations / phases /
delay-spread class, the round trip through the JSON file, a damaged file
read as empty, and the bit masks of window station subsets.  The library is
a fake that records the shapes set, so no kernel runs; timing every shape
on real tables is tests/test_gpu_autotune.py."""
import json

import numpy as np
import pytest

from beampower_b200 import autotune
from beampower_b200.batch import station_mask_words
from beampower_b200.core import REDUCE_MAX, REDUCE_NONE, STORAGE


class FakeLib:
    def __init__(self):
        self.set = []

    def bp_set_kernel_config(self, storage, reduce, config):
        self.set.append((storage, reduce, config))
        return 0


class FakeTable:
    def __init__(self, spread, S=60, P=2):
        self.info = {"max_spread": spread}
        self.n_stations, self.n_phases = S, P


@pytest.fixture
def cache(tmp_path, monkeypatch):
    path = tmp_path / "tune" / "autotune.json"
    monkeypatch.setenv(autotune.CACHE_ENV, str(path))
    lib = FakeLib()
    monkeypatch.setattr(autotune, "load_library", lambda device: lib)
    monkeypatch.setattr(autotune, "_gpu_key", lambda: "NVIDIA B200|148")
    return path, lib


@pytest.mark.parametrize("spread,cls", [(0, 0), (255, 0), (256, 1), (1023, 1), (1024, 2),
                                        (5000, 2)])
def test_spread_classes(cache, spread, cls):
    key = autotune._problem_key(FakeTable(spread), STORAGE["fp16"], "max")
    assert key == f"NVIDIA B200|148|storage={STORAGE['fp16']}|reduce=max|S=60|P=2|spread={cls}"


def test_cache_round_trip_per_table_class(cache):
    path, lib = cache
    fp16 = STORAGE["fp16"]
    autotune._store({autotune._problem_key(FakeTable(300), fp16, "max"):
                     {"config": 2, "ms": {"2": 1.0}}})
    assert json.loads(path.read_text())  # written where the variable points
    # same class (256 <= spread < 1024): applied for the max reduce of fp16
    assert autotune.apply_cached(FakeTable(900), "fp16", "max") == 2
    assert lib.set[-1] == (fp16, REDUCE_MAX, 2)
    # another spread class, stations count, storage or reduce: no entry
    assert autotune.apply_cached(FakeTable(2000), "fp16", "max") is None
    assert autotune.apply_cached(FakeTable(300, S=20), "fp16", "max") is None
    assert autotune.apply_cached(FakeTable(300), "fp32", "max") is None
    assert autotune.apply_cached(FakeTable(300), "fp16", "none") is None
    assert len(lib.set) == 1
    # without a table: any entry of this GPU, storage and reduce
    assert autotune.apply_cached(None, fp16, "max") == 2
    assert autotune.apply_cached(None, "fp32", "none") is None


def test_cache_keeps_other_entries_and_reads_damage_as_empty(cache):
    path, lib = cache
    fp32 = STORAGE["fp32"]
    autotune._store({"other|key": {"config": 1}})
    data = autotune._load()
    data[autotune._problem_key(FakeTable(10), fp32, "none")] = {"config": 8}
    autotune._store(data)
    assert set(autotune._load()) == {"other|key",
                                     autotune._problem_key(FakeTable(10), fp32, "none")}
    assert autotune.apply_cached(FakeTable(10), "fp32", "none") == 8
    assert lib.set[-1] == (fp32, REDUCE_NONE, 8)
    path.write_text("{not json")
    assert autotune._load() == {}
    assert autotune.apply_cached(FakeTable(10), "fp32", "none") is None


def test_station_mask_words():
    w = station_mask_words([0, 5, 31, 32, 69], 70)
    assert w.dtype == np.uint32 and w.shape == (3,)
    assert w[0] == (1 | 1 << 5 | 1 << 31) and w[1] == 1 and w[2] == 1 << 5
    full = station_mask_words(None, 33)
    assert full[0] == 0xFFFFFFFF and full[1] == 1
    assert not station_mask_words([], 40).any()
    with pytest.raises(ValueError):
        station_mask_words([40], 40)
    with pytest.raises(ValueError):
        station_mask_words([-1], 40)
