"""The multi-GPU plumbing (independent replicas) on CPU: two gloo ranks
shard the poses of a batch, synthesise their share with the CPU oracle as a
stand-in for the device, and combine timings the way bench.py does (max over
ranks).  The union of the shards must be the whole batch, each pose once."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from rvsb import replicas


def test_shard_partition():
    for n in (0, 1, 5, 16, 300, 301):
        for world in (1, 2, 3, 8):
            got = [list(replicas.shard(n, r, world)) for r in range(world)]
            flat = [i for g in got for i in g]
            assert flat == list(range(n))
            sizes = [len(g) for g in got]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        replicas.shard(4, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out_dir):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(here)
    sys.path.insert(0, os.path.join(root, "rvs-cuda_b200"))
    sys.path.insert(0, os.path.join(root, "oracle"))
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    from rvsb import replicas as R
    from rvsb import scenes
    import oracle as O
    w, r, _ = R.init(backend="gloo", timeout_s=60)
    assert (w, r) == (world, rank)
    wl = scenes.random_pose_small(n_views=2, w=48, h=32, seed=77)
    targets = [wl.targets[0]] * 5
    mine = R.shard(len(targets), r, w)
    R.barrier(w)
    results = {}
    for i in mine:
        y, u, v = O.synthesize(wl.inputs, wl.planes, targets[i], 5.0)
        results[i] = int(np.asarray(y, np.int64).sum())
    local_time = 0.25 * (r + 1)
    slowest = R.max_over_ranks(local_time, w)
    total = R.sum_over_ranks(len(mine), w)
    R.barrier(w)
    np.save(os.path.join(out_dir, f"rank{r}.npy"),
            np.array([slowest, total] + [results[i] for i in mine] + list(mine), np.float64))
    R.finish(w)


def test_two_gloo_ranks(tmp_path):
    world = 2
    port = _free_port()
    mp.start_processes(_rank_main, args=(world, port, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    r0 = np.load(tmp_path / "rank0.npy")
    r1 = np.load(tmp_path / "rank1.npy")
    assert r0[0] == r1[0] == 0.5          # max over ranks of 0.25, 0.5
    assert r0[1] == r1[1] == 5            # every pose counted once
    # rank 0 owns poses 0-2, rank 1 poses 3-4; identical targets give the
    # identical checksum on both ranks
    n0, n1 = 3, 2
    assert list(r0[2 + n0:]) == [0, 1, 2] and list(r1[2 + n1:]) == [3, 4]
    assert len(set(r0[2:2 + n0]) | set(r1[2:2 + n1])) == 1


def _bcast_main(rank, world, port, out_dir):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(here)
    sys.path.insert(0, os.path.join(root, "rvs-cuda_b200"))
    sys.path.insert(0, os.path.join(root, "oracle"))
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    from rvsb import replicas as R
    from rvsb import scenes
    import oracle as O
    w, r, _ = R.init(backend="gloo", timeout_s=60)
    wl = scenes.random_pose_small(n_views=2, w=48, h=32, seed=78)
    # only rank 0 "reads" the input set; the others receive it
    got = R.broadcast_planes(wl.planes if r == 0 else None, w)
    planes = [tuple(t.numpy().view(np.uint16).reshape(np.asarray(a).shape) for t, a in zip(view, ref))
              for view, ref in zip(got, wl.planes)]
    same = all((a == np.asarray(b)).all() for view, ref in zip(planes, wl.planes) for a, b in zip(view, ref))
    y, u, v = O.synthesize(wl.inputs, planes, wl.targets[0], 5.0)
    R.barrier(w)
    np.save(os.path.join(out_dir, f"b{r}.npy"), np.array([float(same), float(np.asarray(y, np.int64).sum())]))
    R.finish(w)


def test_broadcast_input_set(tmp_path):
    """broadcast_planes: rank 0's input set arrives bit-identical on rank 1,
    and both synthesise the same view from it."""
    world = 2
    port = _free_port()
    mp.start_processes(_bcast_main, args=(world, port, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    b0 = np.load(tmp_path / "b0.npy")
    b1 = np.load(tmp_path / "b1.npy")
    assert b0[0] == 1.0 and b1[0] == 1.0
    assert b0[1] == b1[1]
