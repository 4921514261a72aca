"""One process per GPU: every rank renders its own samples of the same frame
(pixels and samples are independent, path_tracing.cu:30-128) and the ranks'
FP64 films are summed; LVC-BPT runs as replicas the same way, each rank with
its own light-vertex cache.  The only exchange is that film reduction, one
all-reduce of width x height x 16 doubles, which the process group's backend
(NCCL across GPUs) carries.  Timings combine as the maximum over ranks and
work as the sum."""
import torch
import torch.distributed as dist

# The reference's seed of the per-pixel RNG streams (context.cpp:1176-1190).
REFERENCE_SEED = 591842031321323413
_M64 = (1 << 64) - 1


def rank_seed(rank, base=REFERENCE_SEED):
    """Seed of the per-pixel RNG streams of `rank`: rank 0 keeps `base` (so
    one GPU renders exactly the reference's samples), every other rank a
    SplitMix64 hash of base and rank, so the ranks draw independent samples
    and their summed films hold N times the samples instead of N copies."""
    if rank == 0:
        return base
    z = (base + 0x9E3779B97F4A7C15 * rank) & _M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
    z ^= z >> 31
    return z or 1


class _DeviceView:
    """__cuda_array_interface__ over a device allocation of doubles."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "version": 3, "data": (ptr, False)}


def film_tensor(ctx):
    """The context's FP64 film as a CUDA tensor sharing its memory."""
    return torch.as_tensor(_DeviceView(ctx.film_device_ptr(), ctx.height * ctx.width * 16), device="cuda")


def allreduce_film(film, group=None):
    """Sum the ranks' films in place: afterwards every rank holds the film of
    all ranks' samples together."""
    dist.all_reduce(film, op=dist.ReduceOp.SUM, group=group)
    return film


def combine(seconds, units, group=None):
    """(max over ranks of seconds, sum over ranks of units): the job's time
    is its slowest rank's and its work is everyone's."""
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.tensor([float(seconds)], dtype=torch.float64, device=dev)
    u = torch.tensor([float(units)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    dist.all_reduce(u, op=dist.ReduceOp.SUM, group=group)
    return t.item(), u.item()
