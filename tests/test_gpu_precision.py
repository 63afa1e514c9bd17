"""'Precision' P != 1 (SynthesizedView::computeBasicMode,
SynthesizedView.cpp:325-333; write_color, image_writing.cpp:188-190): the
views rasterised at int(0.5 + W*P) x int(0.5 + H*P) with scaled uv and
triangle stretch / P, blended and inpainted at that size, the colour resized
to W x H when written.  The CUDA path against the oracle's restatement."""
import copy

import numpy as np
import pytest
import torch

import oracle as O
import rvsb
from rvsb import scenes
from helpers import assert_parity, gpu_synthesize, to_u16, yuv_planes_torch

pytestmark = pytest.mark.gpu

CASES = [
    dict(n_views=3, w=128, h=64, seed=121),
    dict(n_views=2, w=128, h=64, seed=122, erp_in=True),
    dict(n_views=4, w=160, h=96, seed=123),
    dict(n_views=2, w=128, h=64, seed=124, erp_in=True, erp_out=True),
]


def _params(P, **kw):
    p = rvsb.params(5.0, **kw)
    p.precision = P
    return p


def _oracle(wl, target, P, multispectral=None):
    O.set_precision(P)
    if multispectral:
        O.set_multispectral(True, *multispectral)
    try:
        return O.synthesize(wl.inputs, wl.planes, target, 5.0, want_intermediate=True)
    finally:
        O.set_precision(1.0)
        O.set_multispectral(False)


@pytest.mark.parametrize("case", CASES, ids=lambda c: "-".join(f"{k}{v}" for k, v in c.items()))
@pytest.mark.parametrize("P", [2.0, 1.5, 0.75, 0.5])
def test_precision_matches_oracle(ctx, case, P):
    wl = scenes.random_pose_small(**case)
    target = wl.targets[0]
    yuv, dbg, _ = gpu_synthesize(ctx, wl.inputs, wl.planes, target, 5.0, debug=True, params=_params(P))
    cpu, cq, cc = _oracle(wl, target, P)
    assert dbg["blend_quality"].shape == cq.shape
    np.testing.assert_array_equal(~(dbg["blend_quality"] > 0), ~(cq > 0))
    assert_parity(yuv, cpu)


def test_precision_multispectral(ctx):
    wl = scenes.random_pose_small(n_views=3, w=128, h=64, seed=125)
    target = wl.targets[0]
    yuv, _ = gpu_synthesize(ctx, wl.inputs, wl.planes, target, 5.0, params=_params(2.0, multispectral=(1.0, 8.0)))
    cpu, _, _ = _oracle(wl, target, 2.0, multispectral=(1.0, 8.0))
    assert_parity(yuv, cpu)


def test_precision_differs_from_one(ctx):
    wl = scenes.random_pose_small(n_views=2, w=128, h=64, seed=126)
    t = wl.targets[0]
    a, _ = gpu_synthesize(ctx, wl.inputs, wl.planes, t, 5.0)
    b, _ = gpu_synthesize(ctx, wl.inputs, wl.planes, t, 5.0, params=_params(2.0))
    assert any((x != y).any() for x, y in zip(a, b))


def test_odd_raster_size_rejected(ctx):
    """96 x 54 at P = 1.5 rasterises at 144 x 81: rejected, nothing written."""
    wl = scenes.random_pose_small(n_views=2, w=96, h=54, seed=127)
    with pytest.raises(rvsb.RvsbError) as e:
        gpu_synthesize(ctx, wl.inputs, wl.planes, wl.targets[0], 5.0, params=_params(1.5))
    assert e.value.status == 7
    with pytest.raises(rvsb.RvsbError) as e:
        gpu_synthesize(ctx, wl.inputs, wl.planes, wl.targets[0], 5.0, params=_params(-2.0))
    assert e.value.status == 7


def test_aux_outputs_need_precision_one(ctx):
    wl = scenes.random_pose_small(n_views=2, w=128, h=64, seed=128)
    sc = rvsb.Scene(ctx, wl.inputs)
    for i, p in enumerate(wl.planes):
        sc.upload(i, [np.ascontiguousarray(a, np.uint16) for a in p], on_device=False)
    t = wl.targets[0]
    out = yuv_planes_torch(t.width, t.height)
    mask = torch.zeros(t.height * t.width, dtype=torch.uint8, device="cuda")
    with pytest.raises(rvsb.RvsbError) as e:
        sc.synthesize_aux(t, _params(2.0), out, mask=mask)
    assert e.value.status == 7


def _yuv(out, cam):
    wo, ho = cam.width, cam.height
    return (to_u16(out[0], (ho, wo)), to_u16(out[1], (ho // 2, wo // 2)), to_u16(out[2], (ho // 2, wo // 2)))


def test_precision_batch_and_server(ctx):
    """A batch at P = 2, and a served mix of P = 1, 2 and 0.5 requests,
    give the single synthesis's output bit for bit."""
    wl = scenes.random_pose_small(n_views=3, w=128, h=64, seed=129)
    sc = rvsb.Scene(ctx, wl.inputs)
    for i, p in enumerate(wl.planes):
        sc.upload(i, [np.ascontiguousarray(a, np.uint16) for a in p], on_device=False)
    rng = np.random.default_rng(4)
    cams = []
    for k in range(6):
        c = copy.deepcopy(wl.targets[0])
        c.position[0] += float(rng.uniform(-0.02, 0.02))
        c.rotation[0] += float(rng.uniform(-2, 2))
        cams.append(c)
    Ps = [1.0, 2.0, 0.5, 2.0, 1.0, 0.5]
    alone = []
    for c, P in zip(cams, Ps):
        out = yuv_planes_torch(c.width, c.height)
        sc.synthesize(c, _params(P), out)
        torch.cuda.synchronize()
        alone.append(_yuv(out, c))
    b = rvsb.Batch(sc, 4)
    outs = [yuv_planes_torch(c.width, c.height) for c in cams[:4]]
    b.synthesize(cams[:4], _params(2.0), outs)
    torch.cuda.synchronize()
    for c, o in zip(cams[:4], outs):
        single = yuv_planes_torch(c.width, c.height)
        sc.synthesize(c, _params(2.0), single)
        torch.cuda.synchronize()
        for x, y in zip(_yuv(o, c), _yuv(single, c)):
            np.testing.assert_array_equal(x, y)
    b.close()
    srv = rvsb.Server(ctx, lanes=2, max_batch=4)
    sid = srv.add_scene(sc)
    outs = [yuv_planes_torch(c.width, c.height) for c in cams]
    for c, P, o in zip(cams, Ps, outs):
        srv.submit(sid, c, _params(P), o)
    srv.drain()
    res = srv.poll()
    assert len(res) == len(cams) and all(r[1] == 0 for r in res)
    for c, o, a in zip(cams, outs, alone):
        for x, y in zip(_yuv(o, c), a):
            np.testing.assert_array_equal(x, y)
    srv.close()
