"""The multi-GPU serving router (rvsb/router.py) on CPU: two gloo ranks,
each with a host stand-in for its GPU's serving loop.  Rank 0 routes a
stream of requests least-loaded; the test checks the completion accounting
(every request completed once, on the rank it was routed to, counters
consistent on both sides), that the slower replica receives less work, and
that a request's result does not depend on the replica that served it."""
import json
import os
import socket
import threading
import time
import zlib

import numpy as np
import pytest
import torch.multiprocessing as mp

from rvsb import abi, router


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


class FakeReplica:
    """Host stand-in for one GPU's rvsb_server: a request takes its cost
    estimate times `seconds_per_unit` of simulated service, one at a time in
    arrival order, and its "result" is a checksum of its camera, the same on
    every replica."""

    def __init__(self, seconds_per_unit):
        self.spu = seconds_per_unit
        self.queue = []
        self.busy_until = 0.0
        self.next = 0
        self.results = {}

    def submit(self, scene, camera, params):
        lid = self.next
        self.next += 1
        now = time.monotonic()
        start = max(now, self.busy_until)
        self.busy_until = start + router.request_cost(camera, 1) * self.spu
        self.queue.append((lid, now, start, self.busy_until, scene, bytes(camera)))
        return lid

    def poll(self):
        now = time.monotonic()
        out = []
        keep = []
        for lid, t_sub, t_start, t_done, scene, cam in self.queue:
            if t_done <= now:
                self.results[lid] = zlib.crc32(bytes([scene]) + cam)
                out.append((lid, 0, 1, t_sub, t_start, t_done))
            else:
                keep.append((lid, t_sub, t_start, t_done, scene, cam))
        self.queue = keep
        return out


def _requests(n):
    rng = np.random.default_rng(7)
    reqs = []
    for k in range(n):
        w, h = [(96, 54), (192, 108), (256, 128)][int(rng.integers(0, 3))]
        cam = abi.make_camera(abi.PERSPECTIVE, w, h, position=(float(rng.uniform(-0.1, 0.1)), 0.0, 0.0))
        reqs.append((int(rng.integers(0, 2)), cam))
    return reqs


def _rank_main(rank, world, port, out_dir):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.join(os.path.dirname(here), "rvs-cuda_b200"))
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import rvsb
    from rvsb import replicas as R
    from rvsb import router as RT
    w, r, _ = R.init(backend="gloo", timeout_s=60)
    store = RT.open_store(r, w, timeout_s=60)
    # rank 1's stand-in is three times slower
    replica = FakeReplica(2e-8 * (3.0 if r == 1 else 1.0))
    served = {}
    if r == 0:
        import torch.distributed as dist
        done = []
        # the replica loop of rank 0 runs beside the front end, on its own
        # connection to the store
        worker_store = dist.TCPStore("127.0.0.1", port + 1, w, False)
        t = threading.Thread(target=lambda: done.append(RT.serve_replica(worker_store, 0, replica, timeout_s=60)))
        t.start()
        front = RT.Router(store, w, scene_views=[2, 4])
        p = rvsb.params(5.0)
        routed = []
        for scene, cam in _requests(60):
            rid, rk = front.submit(scene, cam, p)
            routed.append(rk)
            time.sleep(3e-4)
        results = front.finish(timeout_s=60)
        t.join(60)
        served["n"] = done[0]
        served["routed"] = routed
        served["results"] = {str(k): v for k, v in results.items()}
        served["outstanding"] = front.outstanding
        served["counters"] = [store.add(f"nreq/{k}", 0) for k in range(w)] + \
                             [store.add(f"ndone/{k}", 0) for k in range(w)]
    else:
        served["n"] = RT.serve_replica(store, r, replica, timeout_s=60)
    served["local"] = {str(k): v for k, v in replica.results.items()}
    R.barrier(w)
    with open(os.path.join(out_dir, f"rank{r}.json"), "w") as f:
        json.dump(served, f)
    R.finish(w)


def test_router_two_ranks(tmp_path):
    world = 2
    port = _free_port()
    mp.start_processes(_rank_main, args=(world, port, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    r0 = json.load(open(tmp_path / "rank0.json"))
    r1 = json.load(open(tmp_path / "rank1.json"))
    results = {int(k): v for k, v in r0["results"].items()}
    routed = r0["routed"]
    n = len(routed)
    # every request completed once, on the rank it was routed to
    assert sorted(results) == list(range(n))
    assert all(results[i]["rank"] == routed[i] and results[i]["status"] == 0 for i in range(n))
    assert r0["n"] + r1["n"] == n
    assert r0["n"] == routed.count(0) and r1["n"] == routed.count(1)
    nreq0, nreq1, ndone0, ndone1 = r0["counters"]
    assert (nreq0, nreq1) == (routed.count(0), routed.count(1)) == (ndone0, ndone1)
    assert all(abs(x) < 1e-6 for x in r0["outstanding"])
    # least-loaded: the slower replica gets less work, but some
    assert 0 < routed.count(1) < routed.count(0)
    # a request's result is the same whichever replica computed it
    reqs = _requests(n)
    for rank_local, rank_id in ((r0["local"], 0), (r1["local"], 1)):
        ids = [i for i in range(n) if routed[i] == rank_id]
        for lid, rid in enumerate(ids):
            scene, cam = reqs[rid]
            assert rank_local[str(lid)] == zlib.crc32(bytes([scene]) + bytes(cam))


def test_router_single_rank_in_process():
    """World 1 without processes: the router and one replica on one store."""
    import torch.distributed as dist
    port = _free_port()
    store = dist.TCPStore("127.0.0.1", port, 1, True)
    replica = FakeReplica(0.0)
    import rvsb
    front = router.Router(store, 1, scene_views=[3])
    for scene, cam in _requests(10):
        front.submit(0, cam, rvsb.params(5.0))
    client = dist.TCPStore("127.0.0.1", port, 1, False)
    t = threading.Thread(target=lambda: router.serve_replica(client, 0, replica, timeout_s=30))
    t.start()
    res = front.finish(timeout_s=30)
    t.join(30)
    assert sorted(res) == list(range(10)) and all(v["rank"] == 0 for v in res.values())
