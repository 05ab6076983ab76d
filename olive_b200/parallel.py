"""Multi-process plumbing for running the engine on several GPUs of one node.

The traversals in this package do not shard a single graph across GPUs; a
multi-GPU run is a set of replicas (one process per GPU, launched by
torch.distributed.run), each owning whole work units: its own sources for
multi-source BFS, its own instances of a batch, or a full replica of a
single-source run.  Nothing crosses GPUs on the data path; the only
collectives are the timing and counting reductions below (NCCL between GPUs,
gloo on CPU in the tests).
"""
import datetime
import os


def rank_world():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def init(backend="nccl", timeout_s=120, device=None):
    """Join the process group named by the torchrun environment (no-op alone)."""
    import torch.distributed as dist
    _, world, _ = rank_world()
    if world > 1 and not dist.is_initialized():
        kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
        if device is not None:
            kw["device_id"] = device
        dist.init_process_group(backend, **kw)
    return world


def shard(items, rank, world):
    """Contiguous, balanced split of a sequence: shard r of `world`."""
    n = len(items)
    lo = n * rank // world
    hi = n * (rank + 1) // world
    return items[lo:hi]


def _reduce(x, op, device):
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    if dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(x, device="cpu"):
    """Largest value over all ranks (the job time of a multi-GPU step)."""
    import torch.distributed as dist
    return _reduce(x, dist.ReduceOp.MAX, device)


def sum_over_ranks(x, device="cpu"):
    """Sum over all ranks (work units processed by the whole job)."""
    import torch.distributed as dist
    return _reduce(x, dist.ReduceOp.SUM, device)


def finish():
    import torch.distributed as dist
    if dist.is_initialized():
        dist.barrier()
        dist.destroy_process_group()
