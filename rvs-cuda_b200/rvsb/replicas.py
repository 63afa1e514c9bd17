"""Multi-GPU plumbing of the synthesis path: independent replicas.

Views of the virtual cameras are independent of one another (Pipeline.cpp
computes every output frame of every virtual camera from the inputs alone),
so N GPUs run N replicas, each owning a contiguous share of the
(virtual camera, frame) poses.  No synthesis data crosses between ranks;
the collectives are the one-time broadcast of a newly loaded input set from
the rank that read it (broadcast_planes: NCCL over NVLink between GPUs, so
only one process reads the files), the barriers around a timed region and
the reductions of its timings (the slowest rank decides the job time).

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


def broadcast_planes(planes, world, src=0, device=None):
    """Replicates an input set read by rank `src` on every rank.

    planes: on `src`, a list of (Y, U, V, depth) uint16 arrays per view
    (numpy or torch); ignored elsewhere.  Returns the same list on every
    rank as int16 torch tensors holding the uint16 samples, on `device` (the rank's GPU with
    NCCL, the CPU with gloo), ready for Scene.upload.  Shapes travel first,
    then the bytes of each plane."""
    import numpy as np
    import torch
    if world == 1:
        return [[torch.as_tensor(np.ascontiguousarray(a).view(np.int16)) for a in view] for view in planes]
    import torch.distributed as dist
    if device is None:
        device = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else "cpu"
    rank = dist.get_rank()
    if rank == src:
        shapes = [list(np.asarray(a).shape) + [0] * (2 - np.asarray(a).ndim) for view in planes for a in view]
        head = torch.tensor([len(planes)] + [d for s in shapes for d in s], dtype=torch.int64, device=device)
        n = torch.tensor([head.numel()], dtype=torch.int64, device=device)
    else:
        n = torch.zeros(1, dtype=torch.int64, device=device)
    dist.broadcast(n, src)
    if rank != src:
        head = torch.zeros(int(n.item()), dtype=torch.int64, device=device)
    dist.broadcast(head, src)
    nviews = int(head[0].item())
    dims = head[1:].view(-1, 2).tolist()
    out = []
    for v in range(nviews):
        view = []
        for k in range(4):
            h, w = dims[v * 4 + k]
            shape = (h, w) if w else (h,)
            # as bytes: every backend carries uint8 (gloo has no 16-bit integers)
            if rank == src:
                t = torch.as_tensor(np.ascontiguousarray(planes[v][k]).view(np.int16)).to(device).reshape(shape)
            else:
                t = torch.empty(shape, dtype=torch.int16, device=device)
            dist.broadcast(t.view(torch.uint8), src)
            view.append(t)
        out.append(view)
    return out


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
