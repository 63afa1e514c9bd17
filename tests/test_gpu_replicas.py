"""The pose-parallel replicas (rvsb/replicas.py) with the CUDA path on each
rank: two processes joined over gloo share one GPU (this run has one), each
synthesises its shard of the poses through the product's own calls, and
the gathered outputs equal the single-process synthesis of every pose.
The ranks' kernels never wait on one another: the only exchanges are host
collectives after each rank has synchronised its device."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _poses(wl, n):
    import copy
    rng = np.random.default_rng(4)
    out = []
    for _ in range(n):
        c = copy.deepcopy(wl.targets[0])
        c.position[0] += float(rng.uniform(-0.02, 0.02))
        c.rotation[0] += float(rng.uniform(-2, 2))
        out.append(c)
    return out


def _rank_main(rank, world, port, out_dir):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(here)
    sys.path.insert(0, os.path.join(root, "rvs-cuda_b200"))
    sys.path.insert(0, here)
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import torch
    import rvsb
    from rvsb import replicas as R
    from rvsb import scenes
    from helpers import to_u16, yuv_planes_torch
    w, r, _ = R.init(backend="gloo", timeout_s=120)
    wl = scenes.random_pose_small(n_views=2, w=96, h=54, seed=131)
    # rank 0 reads the input set; the others receive it over the group
    got = R.broadcast_planes(wl.planes if r == 0 else None, w)
    ctx = rvsb.Context(0)
    sc = rvsb.Scene(ctx, wl.inputs)
    for i, view in enumerate(got):
        sc.upload(i, [t.numpy().view(np.uint16) for t in view], on_device=False)
    poses = _poses(wl, 5)
    p = rvsb.params(5.0)
    mine = R.shard(len(poses), r, w)
    outs = {}
    for k in mine:
        c = poses[k]
        bufs = yuv_planes_torch(c.width, c.height)
        sc.synthesize(c, p, bufs)
        torch.cuda.synchronize()
        outs[k] = to_u16(bufs[0], (c.height, c.width))
    R.barrier(w)
    total = R.sum_over_ranks(len(mine), w)
    np.savez(os.path.join(out_dir, f"rank{r}.npz"), total=total, **{f"y{k}": v for k, v in outs.items()})
    sc.close()
    ctx.close()
    R.finish(w)


def test_two_replicas_on_one_gpu(tmp_path, ctx):
    import rvsb
    from rvsb import scenes
    from helpers import to_u16, yuv_planes_torch
    import torch
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    z = [np.load(tmp_path / f"rank{r}.npz") for r in range(world)]
    assert int(z[0]["total"]) == int(z[1]["total"]) == 5
    keys = [sorted(int(k[1:]) for k in zr.files if k.startswith("y")) for zr in z]
    assert keys == [[0, 1, 2], [3, 4]]
    wl = scenes.random_pose_small(n_views=2, w=96, h=54, seed=131)
    sc = rvsb.Scene(ctx, wl.inputs)
    for i, pl in enumerate(wl.planes):
        sc.upload(i, [np.ascontiguousarray(a, np.uint16) for a in pl], on_device=False)
    p = rvsb.params(5.0)
    for k, c in enumerate(_poses(wl, 5)):
        bufs = yuv_planes_torch(c.width, c.height)
        sc.synthesize(c, p, bufs)
        torch.cuda.synchronize()
        want = to_u16(bufs[0], (c.height, c.width))
        np.testing.assert_array_equal(z[0 if k < 3 else 1][f"y{k}"], want)
    sc.close()
