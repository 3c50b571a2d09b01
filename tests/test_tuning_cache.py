"""The autotuner's cache file (host logic, CPU).

`steploop.tune_by_bucket` searches one list configuration per size bucket;
with `cache_file` it keeps the results between runs, keyed by GPU model,
library ABI and the kind of search.  The device searches are replaced here by
fakes that record their calls, so the test checks the bookkeeping only: a
second run with the same key searches nothing and hands out the same
tunings, a new bucket is searched alone, and another GPU model or another
search gets entries of its own.
"""

from __future__ import annotations

import json
from types import SimpleNamespace

import pytest


@pytest.fixture
def fake_search(monkeypatch):
    from mdb200 import steploop

    calls = []

    def result(systems):
        atoms = max(s.particle_count for s in systems)
        # a setting that depends on the size, so every bucket gets its own
        return {"verlet_skin": 0.1 + 0.01 * steploop.size_bucket(atoms), "sort_cell": 0.2, "tile_atoms": 8,
                "prune_tiles": 2, "inner_skin": 0.1, "ms_per_step": 1.0, "candidates": 20,
                "systems": len(systems)}

    def autotune(system, state, options=None, steps=200):
        calls.append(("single", system.particle_count))
        return result([system])

    def autotune_batch(systems, states, options=None, steps=200):
        calls.append(("batch", tuple(s.particle_count for s in systems)))
        return result(systems)

    monkeypatch.setattr(steploop, "autotune", autotune)
    monkeypatch.setattr(steploop, "autotune_batch", autotune_batch)
    return calls


def systems_of(sizes):
    return [SimpleNamespace(particle_count=n) for n in sizes], [None] * len(sizes)


def test_second_run_searches_nothing(tmp_path, fake_search):
    from mdb200 import steploop

    path = tmp_path / "tuning.json"
    systems, states = systems_of([2100, 2500, 5000, 9000, 17000, 30000])
    first, _ = steploop.tune_by_bucket(systems, states, batched=True, cache_file=path, gpu="B200")
    searched = len(fake_search)
    assert searched == len({steploop.size_bucket(s.particle_count) for s in systems})
    again, _ = steploop.tune_by_bucket(systems, states, batched=True, cache_file=path, gpu="B200")
    assert len(fake_search) == searched and again == first
    data = json.loads(path.read_text())
    assert list(data) == [steploop.tuning_cache_key("B200", True, 200)]


def test_only_new_buckets_are_searched(tmp_path, fake_search):
    from mdb200 import steploop

    path = tmp_path / "tuning.json"
    systems, states = systems_of([2100, 5000])
    steploop.tune_by_bucket(systems, states, batched=True, cache_file=path, gpu="B200")
    before = len(fake_search)
    bigger, bigger_states = systems_of([2100, 5000, 40000])
    tuning, cache = steploop.tune_by_bucket(bigger, bigger_states, batched=True, cache_file=path, gpu="B200")
    assert fake_search[before:] == [("batch", (40000,))]
    assert len(tuning) == 3 and steploop.size_bucket(40000) in cache


def test_other_gpu_model_or_search_keeps_its_own_entries(tmp_path, fake_search):
    from mdb200 import steploop

    path = tmp_path / "tuning.json"
    systems, states = systems_of([3000, 12000])
    steploop.tune_by_bucket(systems, states, batched=True, cache_file=path, gpu="B200")
    n = len(fake_search)
    steploop.tune_by_bucket(systems, states, batched=True, cache_file=path, gpu="H100")
    assert len(fake_search) == 2 * n
    steploop.tune_by_bucket(systems, states, batched=False, cache_file=path, gpu="B200")
    assert len(fake_search) == 3 * n and all(kind == "single" for kind, _ in fake_search[2 * n:])
    keys = set(json.loads(path.read_text()))
    assert keys == {steploop.tuning_cache_key("B200", True, 200), steploop.tuning_cache_key("H100", True, 200),
                    steploop.tuning_cache_key("B200", False, 200)}


def test_no_file_means_no_cache(tmp_path, fake_search):
    from mdb200 import steploop

    systems, states = systems_of([3000])
    steploop.tune_by_bucket(systems, states, batched=True)
    steploop.tune_by_bucket(systems, states, batched=True)
    assert len(fake_search) == 2
    assert steploop.load_tuning_cache(tmp_path / "absent.json", "any") == {}
