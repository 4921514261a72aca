"""The N > 1 path on CPU: two ranks over gloo exchange their films and
timings exactly as the GPU ranks do over NCCL (vlr_b200.multigpu)."""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        from vlr_b200 import multigpu
        # each rank's film: its own samples of the same 8x8 frame (16 strata)
        rng = np.random.default_rng(100 + rank)
        film = torch.from_numpy(rng.uniform(0, 1, 8 * 8 * 16))
        mine = film.clone()
        multigpu.allreduce_film(film)
        seconds, units = multigpu.combine(0.5 + rank, 1000 * (rank + 1))
        out[rank] = (mine.numpy(), film.numpy(), seconds, units)
    finally:
        dist.destroy_process_group()


def test_two_ranks_sum_films_and_combine_timings():
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
    total = out[0][0] + out[1][0]
    for r in range(world):
        mine, reduced, seconds, units = out[r]
        assert np.allclose(reduced, total, rtol=0, atol=1e-12)
        assert seconds == 1.5            # the slower rank's time
        assert units == 3000.0           # everyone's work
