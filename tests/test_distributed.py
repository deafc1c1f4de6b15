"""The N > 1 path of bench.py on CPU with two gloo ranks: tiles are sharded
across ranks with no overlap (weak scaling, no data collective), timings are
the maximum over ranks, and the reference arm runs on rank 0 only."""

from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out_dir: str) -> None:
    import json

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench

        assert bench.dist_env() == (rank, world, rank)
        slowest = bench.max_over_ranks(1.5 + rank, world, device="cpu")
        tiles = bench.tile_schedule(rank, world, 6)
        gathered = [None] * world
        dist.all_gather_object(gathered, tiles)

        class Args:
            warmup, steps, reference_seconds = 3, 1, 0.1

        if rank != 0:
            # The reference arm does no work and prints nothing off rank 0.
            assert bench.run_reference(Args()) is None
        dist.barrier()
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as handle:
            json.dump({"slowest": slowest, "tiles": gathered}, handle)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_tiles_and_take_the_slowest_time(tmp_path):
    import json

    import torch.multiprocessing as mp

    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    results = [json.loads((tmp_path / f"rank{r}.json").read_text()) for r in range(world)]
    for result in results:
        assert result["slowest"] == 2.5
        per_rank = [set(map(tuple, tiles)) for tiles in result["tiles"]]
        assert len(per_rank[0]) == 6 and len(per_rank[1]) == 6
        assert not per_rank[0] & per_rank[1]
        for tiles in per_rank:
            for row, column in tiles:
                assert row % 128 == 0 and column % 128 == 0
                assert 4 * 128 <= row < 4096 - 4 * 128 and 4 * 128 <= column < 4096 - 4 * 128


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.max_over_ranks(3.25, 1) == 3.25
    assert bench.tile_schedule(0, 1, 3) == bench.tile_schedule(0, 1, 5)[:3]


@pytest.mark.parametrize("world", [2, 4, 8])
def test_schedules_of_all_ranks_are_disjoint(world):
    sys.path.insert(0, str(ROOT))
    import bench

    seen = set()
    for rank in range(world):
        tiles = bench.tile_schedule(rank, world, 10)
        assert len(set(tiles)) == 10
        assert not seen & set(tiles)
        seen |= set(tiles)
