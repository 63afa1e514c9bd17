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


def _frame_buffer(views):
    """The planes of a frame copied into one pinned buffer, back to back in
    the order of the argument (as a loader that reads a frame's files into
    one buffer holds them); returns views of that buffer."""
    buf = torch.empty(sum(t.numel() for planes in views for t in planes), dtype=torch.int16).pin_memory()
    out, off = [], 0
    for planes in views:
        parts = []
        for t in planes:
            part = buf[off:off + t.numel()]
            part.copy_(t)
            parts.append(part)
            off += t.numel()
        out.append(parts)
    return out


@pytest.mark.parametrize("layout", ["frame", "per_view", "mixed"])
def test_adjacent_planes_upload_together(ctx, layout):
    """Input planes adjacent in host memory are uploaded in one copy and a
    YUV420 output that is one buffer is downloaded in one: the whole frame
    in one buffer, each view in its own buffer, and a frame where only some
    planes are adjacent (depth planes apart) give the bytes of separate
    planes, through both the pipelined and the blocking call."""
    wl = scenes.random_pose_small(n_views=3, w=128, h=64, seed=134)
    frames = _frames(wl, 4)
    p = rvsb.params(5.0)
    ref = []
    for planes, cam in frames:
        o = _out(cam)
        ctx.synthesize_host(wl.inputs, planes, cam, p, o)
        ref.append([t.numpy().copy() for t in o])

    def arrange(planes):
        if layout == "frame":
            return _frame_buffer(planes)
        if layout == "per_view":
            return [_frame_buffer([v])[0] for v in planes]
        colour = _frame_buffer([v[:3] for v in planes])
        return [c + [v[3]] for c, v in zip(colour, planes)]

    arranged = [(arrange(planes), cam) for planes, cam in frames]
    hs = rvsb.HostStream(ctx, wl.inputs)
    outs = [_frame_buffer([_out(cam)])[0] for _, cam in frames]
    for (planes, cam), o in zip(arranged, outs):
        hs.submit(planes, cam, p, o)
    hs.join()
    torch.cuda.synchronize()
    for (planes, cam), o, r in zip(arranged, outs, ref):
        for a, b in zip(o, r):
            np.testing.assert_array_equal(a.numpy(), b)
        o2 = _frame_buffer([_out(cam)])[0]
        ctx.synthesize_host(wl.inputs, planes, cam, p, o2)
        for a, b in zip(o2, r):
            np.testing.assert_array_equal(a.numpy(), b)
    hs.close()


def test_device_planes_upload_together(ctx):
    """rvsb_scene_upload from device planes: a view's planes back to back
    in one device buffer (one copy) and in separate tensors give the same
    bytes."""
    wl = scenes.random_pose_small(n_views=2, w=128, h=64, seed=135)
    p = rvsb.params(5.0)
    cam = wl.targets[0]
    results = []
    for together in (False, True):
        sc = rvsb.Scene(ctx, wl.inputs)
        for i, planes in enumerate(wl.planes):
            host = [torch.from_numpy(np.ascontiguousarray(a).view(np.int16)).reshape(-1) for a in planes]
            if together:
                buf = torch.cat(host).cuda()
                dev, off = [], 0
                for t in host:
                    dev.append(buf[off:off + t.numel()])
                    off += t.numel()
            else:
                dev = [t.cuda() for t in host]
            sc.upload(i, dev, on_device=True)
        out = [t.cuda() for t in _out(cam)]
        sc.synthesize(cam, p, out)
        torch.cuda.synchronize()
        results.append([t.cpu().numpy() for t in out])
        sc.close()
    for a, b in zip(*results):
        np.testing.assert_array_equal(a, b)
