"""Pipelined host frames (rvsb_host_stream_*): the uploads of one frame,
the synthesis of the previous one and the download of the one before
overlap on three streams.  Every frame's output is bit-identical to the
blocking rvsb_synthesize_host call on the same inputs."""
import copy

import numpy as np
import pytest
import torch

import rvsb
from rvsb import scenes

pytestmark = pytest.mark.gpu


def _pinned(a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int16)).reshape(-1).pin_memory()


def _frames(wl, n):
    """n input frames: the workload's planes with luma shifted per frame,
    and one pose per frame."""
    rng = np.random.default_rng(17)
    frames = []
    for k in range(n):
        planes = []
        for y, u, v, d in wl.planes:
            y2 = np.clip(y.astype(np.int32) + 5 * k, 0, 1023).astype(np.uint16)
            planes.append([_pinned(a) for a in (y2, u, v, d)])
        cam = copy.deepcopy(wl.targets[0])
        cam.position[0] += float(rng.uniform(-0.02, 0.02))
        cam.rotation[0] += float(rng.uniform(-2, 2))
        frames.append((planes, cam))
    return frames


def _out(cam):
    wo, ho = cam.width, cam.height
    return [torch.zeros(n, dtype=torch.int16).pin_memory() for n in (wo * ho, wo * ho // 4, wo * ho // 4)]


@pytest.mark.parametrize("case", [dict(n_views=3, w=128, h=64, seed=131),
                                  dict(n_views=2, w=128, h=64, seed=132, erp_in=True)])
def test_host_stream_matches_blocking_call(ctx, case):
    wl = scenes.random_pose_small(**case)
    frames = _frames(wl, 7)
    p = rvsb.params(5.0)
    ref = []
    for planes, cam in frames:
        o = _out(cam)
        ctx.synthesize_host(wl.inputs, planes, cam, p, o)
        ref.append([t.numpy().copy() for t in o])
    hs = rvsb.HostStream(ctx, wl.inputs)
    outs = [_out(cam) for _, cam in frames]
    tickets = [hs.submit(planes, cam, p, o) for (planes, cam), o in zip(frames, outs)]
    assert tickets == list(range(len(frames)))
    for t in reversed(tickets):  # waiting on an old ticket after newer ones is allowed
        hs.wait(t)
    for o, r in zip(outs, ref):
        for a, b in zip(o, r):
            np.testing.assert_array_equal(a.numpy(), b)
    with pytest.raises(rvsb.RvsbError):
        hs.wait(len(frames))
    hs.close()


def test_host_stream_join_and_reuse(ctx):
    """Two output buffers reused in turn, completion through join on a
    caller stream; precision and multispectral parameters pass through."""
    wl = scenes.random_pose_small(n_views=3, w=128, h=64, seed=133)
    frames = _frames(wl, 6)
    p = rvsb.params(5.0, multispectral=(1.0, 8.0))
    p.precision = 2.0
    hs = rvsb.HostStream(ctx, wl.inputs)
    bufs = [_out(frames[0][1]), _out(frames[0][1])]
    stream = torch.cuda.Stream()
    got = []
    for k, (planes, cam) in enumerate(frames):
        t = hs.submit(planes, cam, p, bufs[k % 2], stream=stream)
        if k >= 1:
            hs.wait(t - 1)
            got.append([x.numpy().copy() for x in bufs[(k - 1) % 2]])
    hs.join(stream)
    stream.synchronize()
    got.append([x.numpy().copy() for x in bufs[(len(frames) - 1) % 2]])
    for (planes, cam), g in zip(frames, got):
        o = _out(cam)
        ctx.synthesize_host(wl.inputs, planes, cam, p, o)
        for a, b in zip(g, o):
            np.testing.assert_array_equal(a, b.numpy())
    hs.close()
