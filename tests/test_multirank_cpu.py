"""The N > 1 host paths on CPU: world_size-2 gloo process groups stand in for
two GPUs (one process each).  Covered: the deal of batched replicas to ranks
by balanced site count, the end-of-run gather of per-replica scalars, and the
bench's max-over-ranks timing reduction and barrier."""
import json
import os
import socket

import pytest

from md_engine_b200.replicas import shard_by_sites


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_shard_by_sites_covers_every_replica_once_and_balances():
    import numpy as np

    rng = np.random.default_rng(5)
    sites = [int(4 * m) for m in np.exp(rng.uniform(np.log(256), np.log(2048), 128))]
    for world in (1, 2, 3, 8):
        parts = shard_by_sites(sites, world)
        flat = sorted(r for p in parts for r in p)
        assert flat == list(range(len(sites)))
        loads = [sum(sites[r] for r in p) for p in parts]
        # greedy largest-first: the spread is at most one replica
        assert max(loads) - min(loads) <= max(sites)
        assert all(p == sorted(p) for p in parts)
    assert shard_by_sites(sites, 4) == shard_by_sites(list(sites), 4)  # deterministic
    with pytest.raises(ValueError):
        shard_by_sites(sites, 0)


def _rank_main(rank, world, port, outdir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    os.environ["RANK"] = str(rank)
    os.environ["WORLD_SIZE"] = str(world)
    import datetime

    import torch.distributed as dist

    import bench
    from md_engine_b200.replicas import gather_replica_scalars, shard_by_sites

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    sites = [4 * m for m in (256, 2048, 700, 300, 1500, 900, 1100, 256, 400)]
    mine = shard_by_sites(sites, world)[rank]
    temps = gather_replica_scalars(dist, mine, [1000.0 + r for r in mine], len(sites))
    slowest = bench.reduce_max(dist, 1.5 + rank)
    bench.barrier(dist)
    with open(os.path.join(outdir, f"rank{rank}.json"), "w") as f:
        json.dump({"mine": mine, "temps": temps, "max": slowest}, f)
    dist.destroy_process_group()


def test_two_rank_gloo_gather_reduce_barrier(tmp_path):
    import torch.multiprocessing as mp

    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    mine = [r["mine"] for r in res]
    assert sorted(mine[0] + mine[1]) == list(range(9)) and not set(mine[0]) & set(mine[1])
    for r in res:
        assert r["temps"] == [1000.0 + k for k in range(9)]  # every replica, in replica order
        assert r["max"] == 2.5  # the slower rank's time on every rank
