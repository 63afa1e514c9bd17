"""Multi-GPU plumbing of the synthesis path: independent replicas.

Views of the virtual cameras are independent of one another (Pipeline.cpp
computes every output frame of every virtual camera from the inputs alone),
so N GPUs run N replicas, each owning a contiguous share of the
(virtual camera, frame) poses.  No data crosses between ranks; the only
collectives are the barriers around a timed region and the reductions of
its timings (the slowest rank decides the job time).

One process per GPU, launched by torch.distributed.run; RANK, LOCAL_RANK,
WORLD_SIZE and MASTER_ADDR/PORT come from the environment.
"""
import datetime
import os


def env():
    """(world, rank, local_rank) from the launcher's environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend=None, timeout_s=300):
    """Joins the process group when WORLD_SIZE > 1 (NCCL when a device is
    present, else gloo).  Returns (world, rank, local_rank)."""
    world, rank, local = env()
    if world > 1:
        import torch
        import torch.distributed as dist
        if not dist.is_initialized():
            if backend is None:
                backend = "nccl" if torch.cuda.is_available() else "gloo"
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return world, rank, local


def shard(n, rank, world):
    """The contiguous range of the n poses owned by `rank`: sizes differ by
    at most one, lower ranks take the extra ones."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def _reduce(x, op, world):
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(x, world):
    if world == 1:
        return float(x)
    import torch.distributed as dist
    return _reduce(x, dist.ReduceOp.MAX, world)


def sum_over_ranks(x, world):
    if world == 1:
        return float(x)
    import torch.distributed as dist
    return _reduce(x, dist.ReduceOp.SUM, world)


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def finish(world):
    if world > 1:
        import torch.distributed as dist
        if dist.is_initialized():
            dist.destroy_process_group()
