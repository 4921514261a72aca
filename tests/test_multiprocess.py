"""The N > 1 path on CPU: two ranks over gloo exchange their films and
timings exactly as the GPU ranks do over NCCL (vlr_b200.multigpu), and each
rank renders its own samples: a rank's per-pixel RNG streams come from its
own seed, so the summed film holds twice the samples, not two copies."""
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
        seed = multigpu.rank_seed(rank)
        from oracle import ref
        if ref.available():
            # each rank's film: its own samples of the same 8x8 Cornell frame,
            # rendered by the CPU oracle from the rank's seed
            from vlr_b200 import scenes
            desc = scenes.cornell_box_desc(8, 8)
            f, _, _ = ref.pt_render(scenes.flatten_desc(desc), desc["camera"], 8, 8, 4, 8,
                                    rng_states=ref.seed_states(64, seed), threads=1)
            film = torch.from_numpy(f.reshape(-1).copy())
        else:
            rng = np.random.default_rng(seed & 0xFFFFFFFF)
            film = torch.from_numpy(rng.uniform(0, 1, 8 * 8 * 16))
        mine = film.clone()
        multigpu.allreduce_film(film)
        seconds, units = multigpu.combine(0.5 + rank, 1000 * (rank + 1))
        out[rank] = (seed, mine.numpy(), film.numpy(), seconds, units)
    finally:
        dist.destroy_process_group()


def test_two_ranks_sum_films_and_combine_timings():
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
    from vlr_b200 import multigpu
    assert out[0][0] == multigpu.REFERENCE_SEED          # one GPU renders the reference's samples
    assert out[0][0] != out[1][0]                         # ranks draw independent samples
    assert not np.array_equal(out[0][1], out[1][1])       # so their films differ
    total = out[0][1] + out[1][1]
    for r in range(world):
        seed, mine, reduced, seconds, units = out[r]
        assert np.allclose(reduced, total, rtol=0, atol=1e-12)
        assert seconds == 1.5            # the slower rank's time
        assert units == 3000.0           # everyone's work


def test_rank_seeds_are_distinct():
    from vlr_b200 import multigpu
    seeds = [multigpu.rank_seed(r) for r in range(64)]
    assert len(set(seeds)) == 64 and all(0 < s < 2 ** 64 for s in seeds)
