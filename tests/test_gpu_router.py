"""The serving router (rvsb/router.py) over a real rvsb_server on one GPU,
world size 1 in one process: requests routed through the store, served by
ServerReplica, each output bit-identical to the per-view call for the same
camera.  (Several replicas on several GPUs are covered on CPU by
test_router_gloo.py; this run has one GPU.)"""
import copy
import socket
import threading

import numpy as np
import pytest

import rvsb
from rvsb import router, scenes
from helpers import to_u16, yuv_planes_torch

pytestmark = pytest.mark.gpu


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_router_with_server_replica(ctx):
    import torch
    import torch.distributed as dist
    wls = [scenes.random_pose_small(n_views=2, w=96, h=54, seed=141),
           scenes.random_pose_small(n_views=3, w=128, h=64, seed=142, erp_in=True)]
    scs = []
    for wl in wls:
        sc = rvsb.Scene(ctx, wl.inputs)
        for i, p in enumerate(wl.planes):
            sc.upload(i, [np.ascontiguousarray(a, np.uint16) for a in p], on_device=False)
        scs.append(sc)
    srv = rvsb.Server(ctx, lanes=2, max_batch=4)
    ids = [srv.add_scene(sc) for sc in scs]
    outputs = {}
    replica = router.ServerReplica(srv, ids, lambda cam: yuv_planes_torch(cam.width, cam.height),
                                   on_done=lambda lid, bufs: outputs.__setitem__(lid, bufs))
    order = []  # the server's ids in the order the requests reached the replica
    submit = replica.submit
    replica.submit = lambda *a: order.append(submit(*a)) or order[-1]
    port = _free_port()
    store = dist.TCPStore("127.0.0.1", port, 1, True)
    client = dist.TCPStore("127.0.0.1", port, 1, False)
    served = []
    t = threading.Thread(target=lambda: served.append(router.serve_replica(client, 0, replica, timeout_s=120)))
    t.start()
    front = router.Router(store, 1, scene_views=[len(wl.inputs) for wl in wls])
    p = rvsb.params(5.0)
    rng = np.random.default_rng(3)
    cams = []
    for k in range(12):
        s = k % 2
        c = copy.deepcopy(wls[s].targets[0])
        c.position[0] += float(rng.uniform(-0.02, 0.02))
        c.rotation[0] += float(rng.uniform(-2, 2))
        cams.append((s, c))
        front.submit(s, c, p)
    res = front.finish(timeout_s=120)
    t.join(120)
    assert served == [12] and sorted(res) == list(range(12)) and all(v["status"] == 0 for v in res.values())
    torch.cuda.synchronize()
    # with one replica, request k is the k-th to reach it
    for k, (s, c) in enumerate(cams):
        alone = yuv_planes_torch(c.width, c.height)
        scs[s].synthesize(c, p, alone)
        torch.cuda.synchronize()
        got = outputs[order[k]]
        for a, b, shape in zip(got, alone, ((c.height, c.width), (c.height // 2, c.width // 2),
                                            (c.height // 2, c.width // 2))):
            np.testing.assert_array_equal(to_u16(a, shape), to_u16(b, shape))
    srv.close()
    for sc in scs:
        sc.close()
