"""Multi-GPU: replicas, one process per GPU (launched by torchrun).

The arena sweep does not shard: a step's growth and coset offsets are dense high-bit XOR masks, so splitting the
arena by address bits would need an all-to-all after every step.  Each GPU therefore runs its own engine on its own
items (strings, samples, instances), and the only collectives are host-side bookkeeping: a barrier around timed
regions, the maximum of the ranks' times, and gathering the ranks' results.  With the gloo backend the same code runs
on CPU processes (tests).
"""
import datetime
import os


def init(backend=None, timeout_s=300):
    """(rank, world, local_rank) from the torchrun environment; joins the process group when world > 1.
    backend: 'nccl' when CUDA is available, else 'gloo' (unless given)."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        if not dist.is_initialized():
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return rank, world, local


def _device():
    import torch
    import torch.distributed as dist
    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    """The largest of the ranks' values (the job's time is the slowest replica's)."""
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def item_range(first, count, rank):
    """Items of one replica under weak scaling: every rank takes `count` items, rank r the block after r's
    predecessors (sample indices first + r * count ...), so the replicas' seeds never overlap."""
    start = int(first) + int(rank) * int(count)
    return start, int(count)


def gather(obj, world):
    """Every rank's object, in rank order, on every rank (host-side results: bits, log2 Pr)."""
    if world == 1:
        return [obj]
    import torch.distributed as dist
    out = [None] * world
    dist.all_gather_object(out, obj)
    return out


def finish(world):
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
