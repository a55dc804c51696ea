"""Multi-rank host logic on CPU: two gloo ranks (127.0.0.1) run the same rank helpers that
bench.py uses over NCCL (kassiopeia_b200/ranks.py): disjoint reproducible point blocks, a
barrier, and the max over ranks of a per-rank time."""

import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from kassiopeia_b200 import ranks as RK

        P = RK.rank_points(500, rank)
        blocks = [None] * world
        dist.all_gather_object(blocks, P)
        RK.barrier(dist)
        t = RK.max_over_ranks(0.25 + rank, dist)
        np.save(os.path.join(out, f"rank{rank}.npy"),
                np.array([t, float(all(np.array_equal(blocks[r], RK.rank_points(500, r)) for r in range(world))),
                          float(min(np.min(np.abs(blocks[a][:, None, :] - blocks[b][None, :, :]).sum(-1))
                                    for a in range(world) for b in range(world) if a < b))]))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks(tmp_path):
    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    for r in range(world):
        t, same, sep = np.load(tmp_path / f"rank{r}.npy")
        assert t == 0.25 + (world - 1)  # every rank sees the slowest rank's time
        assert same == 1.0              # every rank's block is the seeded block of that rank
        assert sep > 0.0                # blocks are disjoint (no shared point)
