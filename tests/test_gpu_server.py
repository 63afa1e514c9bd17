"""The serving loop (rvsb_server_*): requests on resident scenes with
continuous batching.  Each request's output is bit-identical whether it ran
alone or in a mix of scenes, sizes and projections launched together; the
HBM budget bounds what runs at once."""
import copy
import time

import numpy as np
import pytest

import rvsb
from rvsb import abi, scenes
from helpers import to_u16, yuv_planes_torch

pytestmark = pytest.mark.gpu


def _upload(ctx, wl):
    sc = rvsb.Scene(ctx, wl.inputs)
    for i, p in enumerate(wl.planes):
        sc.upload(i, [np.ascontiguousarray(a, np.uint16) for a in p], on_device=False)
    return sc


def _yuv(out, cam):
    wo, ho = cam.width, cam.height
    return (to_u16(out[0], (ho, wo)), to_u16(out[1], (ho // 2, wo // 2)), to_u16(out[2], (ho // 2, wo // 2)))


def _requests(wla, wlb, n):
    """n requests alternating between two scenes, with mixed output sizes and
    an equirectangular output now and then."""
    rng = np.random.default_rng(9)
    reqs = []
    for k in range(n):
        which = k % 2
        base = (wla if which == 0 else wlb).targets[0]
        c = copy.deepcopy(base)
        c.position[0] += float(rng.uniform(-0.02, 0.02))
        c.position[1] += float(rng.uniform(-0.02, 0.02))
        c.rotation[0] += float(rng.uniform(-3, 3))
        if k % 5 == 2:
            c.width, c.height = base.width // 4 * 2, base.height // 4 * 2
            c.focal[0] *= 0.5
            c.focal[1] *= 0.5
            c.principle_point[0] *= 0.5
            c.principle_point[1] *= 0.5
        if k % 7 == 3:
            c = abi.make_camera(abi.EQUIRECTANGULAR, 128, 64, tuple(c.position), (float(rng.uniform(-30, 30)), 0, 0),
                                (0.3, 20.0))
        reqs.append((which, c))
    return reqs


def test_server_alone_vs_mix(ctx):
    import torch
    wla = scenes.random_pose_small(n_views=3, w=96, h=54, seed=61)
    wlb = scenes.random_pose_small(n_views=2, w=128, h=64, seed=62, erp_in=True)
    sa, sb = _upload(ctx, wla), _upload(ctx, wlb)
    p = rvsb.params(5.0)
    reqs = _requests(wla, wlb, 24)
    alone = []
    for which, c in reqs:
        out = yuv_planes_torch(c.width, c.height)
        (sa if which == 0 else sb).synthesize(c, p, out)
        torch.cuda.synchronize()
        alone.append(_yuv(out, c))
    srv = rvsb.Server(ctx, lanes=3, max_batch=4)
    ida, idb = srv.add_scene(sa), srv.add_scene(sb)
    srv.reserve(ida, 128, 64)
    srv.reserve(idb, 128, 64)
    for rep in range(2):
        outs = [yuv_planes_torch(c.width, c.height) for _, c in reqs]
        ids = [srv.submit(ida if which == 0 else idb, c, p, o) for (which, c), o in zip(reqs, outs)]
        srv.drain()
        res = {r[0]: r for r in srv.poll()}
        assert sorted(res) == sorted(ids)
        assert all(r[1] == 0 for r in res.values())
        assert max(r[2] for r in res.values()) > 1, "no request ran in a mix"
        for (which, c), o, a in zip(reqs, outs, alone):
            for x, y in zip(_yuv(o, c), a):
                np.testing.assert_array_equal(x, y)
    srv.close()


def test_server_budget_admission(ctx):
    import torch
    wl = scenes.random_pose_small(n_views=2, w=96, h=54, seed=63)
    sc = _upload(ctx, wl)
    p = rvsb.params(5.0)
    probe = rvsb.Server(ctx, lanes=1, max_batch=1)
    sid = probe.add_scene(sc)
    probe.close()
    # a budget that fits one request of this size, not two
    need = None
    for budget_guess in (1 << 20, 2 << 20, 4 << 20, 8 << 20):
        srv = rvsb.Server(ctx, lanes=2, max_batch=4, hbm_budget=budget_guess)
        sid = srv.add_scene(sc)
        c = wl.targets[0]
        try:
            srv.submit(sid, c, p, yuv_planes_torch(c.width, c.height))
        except rvsb.RvsbError as e:
            assert e.status == 4  # RVSB_E_OOM_BUDGET
            srv.close()
            continue
        srv.drain()
        srv.poll()
        need = budget_guess
        break
    assert need is not None
    outs = [yuv_planes_torch(c.width, c.height) for _ in range(6)]
    for o in outs:
        srv.submit(sid, wl.targets[0], p, o)
    srv.drain()
    res = srv.poll()
    assert len(res) == 6 and all(r[1] == 0 for r in res)
    # with room for one request at a time, nothing ran together
    assert max(r[2] for r in res) == 1
    ref = yuv_planes_torch(c.width, c.height)
    sc.synthesize(wl.targets[0], p, ref)
    torch.cuda.synchronize()
    for o in outs:
        for x, y in zip(_yuv(o, c), _yuv(ref, c)):
            np.testing.assert_array_equal(x, y)
    srv.close()


def test_server_open_loop_times(ctx):
    wl = scenes.random_pose_small(n_views=2, w=96, h=54, seed=64)
    sc = _upload(ctx, wl)
    p = rvsb.params(5.0)
    srv = rvsb.Server(ctx, lanes=2, max_batch=4)
    sid = srv.add_scene(sc)
    srv.reserve(sid, 96, 54)
    c = wl.targets[0]
    outs = [yuv_planes_torch(c.width, c.height) for _ in range(8)]
    rng = np.random.default_rng(3)
    for k in range(40):
        srv.submit(sid, c, p, outs[k % 8])
        time.sleep(float(rng.exponential(0.001)))
    srv.drain()
    res = srv.poll()
    assert len(res) == 40
    for _, st, bs, t0, t1, t2 in res:
        assert st == 0 and 1 <= bs <= 4
        assert t0 <= t1 <= t2
    srv.close()
