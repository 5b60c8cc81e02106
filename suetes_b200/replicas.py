"""Replica parallelism: one process per GPU, independent members, no
data-path collective.

The SISL step of one member does not shard across GPUs in this build (a
horizontal decomposition would need halo exchanges per Arnoldi step); the
parallel unit is the member (an ensemble member or a replica of the whole
run).  Ranks share nothing but the timing reduction: every multi-GPU number
is the maximum over ranks of device-timed work.  ``shard`` assigns members
to ranks when an ensemble is split instead of replicated.
"""

import datetime
import os

import torch


def env():
    """(world, rank, local_rank) from the torchrun environment (1, 0, 0 alone)."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend=None, timeout_s=300):
    """Join the process group when WORLD_SIZE > 1 (nccl with CUDA, else gloo);
    returns (world, rank, local_rank)."""
    world, rank, local = env()
    if torch.cuda.is_available():
        torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        if not dist.is_initialized():
            if backend is None:
                backend = "nccl" if torch.cuda.is_available() else "gloo"
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return world, rank, local


def _device():
    import torch.distributed as dist
    return torch.device("cuda") if dist.get_backend() == "nccl" else torch.device("cpu")


def max_over_ranks(x, world):
    """Maximum of a scalar over the ranks (the timing rule for multi-GPU numbers)."""
    if world == 1:
        return float(x)
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def shard(n_units, rank, world):
    """Contiguous, balanced block of ``range(n_units)`` for ``rank``: every
    unit on exactly one rank, sizes differing by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must lie in [0, world)")
    base, extra = divmod(n_units, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def finalize(world):
    if world > 1:
        import torch.distributed as dist
        if dist.is_initialized():
            dist.destroy_process_group()
