"""The autotuner's cache (host side, no GPU): a stored choice is applied for
the same kind of workload, entries of a library built from other kernel
sources are ignored, and a damaged cache file is treated as empty."""
import json
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


@pytest.fixture()
def tuner(tmp_path, monkeypatch):
    from libsupermesh_b200 import autotune, build

    build.build()
    import libsupermesh_b200 as lsm

    monkeypatch.setenv("LIBSUPERMESH_TUNING_CACHE", str(tmp_path / "tuning.json"))
    names = ("query_block", "tri_blocks_per_sm", "leaf_bucket")
    before = {n: lsm.get_option(n) for n in names}
    yield autotune, lsm
    for n, v in before.items():
        lsm.set_option(n, v)


def test_stored_choice_is_applied(tuner):
    autotune, lsm = tuner
    setting = {"query_block": 64, "tri_blocks_per_sm": 8}
    db = {autotune._key(3, 1000, 2000): {"setting": setting, "ms": 1.0, "source": autotune._source_hash()}}
    autotune.cache_path().write_text(json.dumps(db))
    assert autotune.apply_cached(3, 1000, 2000) == setting
    assert lsm.get_option("query_block") == 64
    # the same size class (rounded log2 of the element count) shares the entry
    assert autotune.apply_cached(3, 1100, 1900) == setting
    # another dimension has none
    assert autotune.apply_cached(2, 1000, 2000) is None


def test_stale_and_damaged_entries_are_ignored(tuner):
    autotune, lsm = tuner
    lsm.set_option("query_block", 128)
    db = {autotune._key(2, 500, 500): {"setting": {"query_block": 256}, "ms": 1.0, "source": "0" * 16}}
    autotune.cache_path().write_text(json.dumps(db))
    assert autotune.apply_cached(2, 500, 500) is None
    assert lsm.get_option("query_block") == 128
    autotune.cache_path().write_text("{not json")
    assert autotune.apply_cached(2, 500, 500) is None


def test_store_round_trip(tuner):
    autotune, _ = tuner
    db = {"k": {"setting": {"query_block": 64}}}
    autotune._store(db)
    assert autotune._load() == db
    assert not autotune.cache_path().with_suffix(".tmp").exists()
