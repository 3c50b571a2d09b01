"""Sharding the batched ensemble over ranks (host logic, CPU, gloo).

The reference has no multi-device code; the unit that shards is the
independent system.  These tests cover the longest-processing-time split and
the per-system report gather with two gloo ranks on the CPU; the GPU side of a
rank is the same batched engine the single-GPU tests cover.
"""

from __future__ import annotations

import itertools
import json
import os
import socket

import numpy as np
import pytest

from mdb200 import shard


def best_split(costs, parts):
    best = float("inf")
    for labels in itertools.product(range(parts), repeat=len(costs)):
        loads = [0.0] * parts
        for c, g in zip(costs, labels):
            loads[g] += c
        best = min(best, max(loads))
    return best


@pytest.mark.parametrize("parts", [2, 3])
def test_lpt_is_within_its_bound_of_the_best_split(parts):
    rng = np.random.default_rng(parts)
    for _ in range(20):
        costs = rng.integers(1, 100, size=9).tolist()
        groups = shard.lpt_partition(costs, parts)
        assert sorted(i for g in groups for i in g) == list(range(len(costs)))
        worst = max(sum(costs[i] for i in g) for g in groups)
        assert worst <= (4 / 3 - 1 / (3 * parts)) * best_split(costs, parts) + 1e-9


def test_lpt_balances_the_ensemble_sizes():
    """Atom counts drawn like the 64-system ensemble's (log-uniform 2,000 to
    30,000): every split up to 8 ranks is within 3% of the mean load."""
    rng = np.random.default_rng(1)
    sizes = np.exp(rng.uniform(np.log(2000), np.log(30000), size=64)).astype(int).tolist()
    for world in (1, 2, 4, 8):
        groups = shard.lpt_partition(sizes, world)
        loads = [sum(sizes[i] for i in g) for g in groups]
        assert max(loads) <= 1.03 * sum(sizes) / world, (world, loads)
        assert groups == shard.lpt_partition(sizes, world)  # the same on every rank
        assert all(g == sorted(g) for g in groups)


def test_rank_share_rejects_a_rank_outside_the_world():
    with pytest.raises(ValueError):
        shard.rank_share([1, 2, 3], 2, 2)
    with pytest.raises(ValueError):
        shard.lpt_partition([1, 2], 0)


def _rank_main(rank, world, port, costs, out_dir):
    import torch.distributed as dist

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        mine = shard.rank_share(costs, rank, world)
        reports = {i: {"rank": rank, "atoms": costs[i]} for i in mine}
        merged = shard.gather_by_system(reports, world)
        # a system claimed by both ranks is refused on every rank, after the
        # gather has completed, so no rank is left waiting
        try:
            shard.gather_by_system({0: {"rank": rank}}, world)
            duplicate = "accepted"
        except RuntimeError as exc:
            duplicate = str(exc)
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"share": mine, "merged": {str(k): v for k, v in merged.items()}, "duplicate": duplicate}, f)
    finally:
        dist.destroy_process_group()


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_shard_the_ensemble_and_gather_every_report(tmp_path):
    import torch.multiprocessing as mp

    rng = np.random.default_rng(7)
    costs = np.exp(rng.uniform(np.log(2000), np.log(30000), size=64)).astype(int).tolist()
    mp.spawn(_rank_main, args=(2, _free_port(), costs, str(tmp_path)), nprocs=2, join=True)
    out = [json.loads((tmp_path / f"rank{r}.json").read_text()) for r in range(2)]
    assert sorted(out[0]["share"] + out[1]["share"]) == list(range(64))
    assert out[0]["merged"] == out[1]["merged"]
    merged = out[0]["merged"]
    assert sorted(int(k) for k in merged) == list(range(64))
    for r in range(2):
        assert all(merged[str(i)]["rank"] == r for i in out[r]["share"])
        assert "reported by two ranks" in out[r]["duplicate"]
