"""The multi-rank host logic of the bench on CPU: two gloo ranks (no GPU).

The template-matching path shards by image with no exchange between ranks;
the only collectives are the barrier and the max over ranks of the timed
interval. Both run here over gloo on 127.0.0.1."""
import os
import socket

import pytest

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, items, out_dir):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        mine = bench.shard(items, rank, world)
        # each rank reports a different "time"; every rank must see the max
        t = bench.allreduce_max(10.0 * (rank + 1))
        bench.barrier()
        with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
            f.write(repr((mine, t)))
    finally:
        dist.destroy_process_group()


def test_shard_partitions_items():
    items = list(range(16))
    for world in (1, 2, 3, 4, 8):
        shares = [bench.shard(items, r, world) for r in range(world)]
        flat = sorted(x for sh in shares for x in sh)
        assert flat == items
        sizes = [len(sh) for sh in shares]
        assert max(sizes) - min(sizes) <= 1


def test_two_gloo_ranks_shard_and_take_the_max(tmp_path):
    import torch.multiprocessing as mp
    world, items = 2, list(range(16))
    mp.spawn(_rank_main, args=(world, _free_port(), items, str(tmp_path)), nprocs=world,
             join=True)
    got = [eval(open(tmp_path / f"rank{r}.txt").read()) for r in range(world)]
    assert sorted(x for mine, _ in got for x in mine) == items
    assert all(t == pytest.approx(20.0) for _, t in got)
