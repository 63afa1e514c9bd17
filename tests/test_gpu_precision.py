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


@pytest.mark.parametrize("w,h,P", [(96, 54, 1.5), (98, 54, 1.5), (64, 36, 0.75), (100, 50, 0.9)],
                         ids=["144x81", "147x81", "48x27", "90x45"])
def test_odd_raster_size(ctx, w, h, P):
    """Raster sizes with an odd side (SynthesizedView.cpp:324-331 allows
    any): the 2x2 blocks of the tile writer, the inpainting fill and the
    multispectral blend end in partial blocks.  Hole mask identical to the
    oracle's, output at parity, per-view call and multispectral."""
    wl = scenes.random_pose_small(n_views=2, w=w, h=h, seed=127)
    target = wl.targets[0]
    target.rotation[0] += 4.0  # border holes reach the odd edge
    yuv, dbg, _ = gpu_synthesize(ctx, wl.inputs, wl.planes, target, 5.0, debug=True, params=_params(P))
    cpu, cq, _ = _oracle(wl, target, P)
    rw, rh = int(np.float32(0.5) + np.float32(w) * np.float32(P)), int(np.float32(0.5) + np.float32(h) * np.float32(P))
    assert cq.shape == (rh, rw) and (rw % 2 or rh % 2)
    np.testing.assert_array_equal(~(dbg["blend_quality"] > 0), ~(cq > 0))
    assert (~(cq > 0)).any()
    assert_parity(yuv, cpu)
    plain, _ = gpu_synthesize(ctx, wl.inputs, wl.planes, target, 5.0, params=_params(P))
    for a, b in zip(plain, yuv):
        np.testing.assert_array_equal(a, b)
    ms, _ = gpu_synthesize(ctx, wl.inputs, wl.planes, target, 5.0, params=_params(P, multispectral=(1.0, 8.0)))
    assert_parity(ms, _oracle(wl, target, P, multispectral=(1.0, 8.0))[0])


def test_invalid_precision_rejected(ctx):
    wl = scenes.random_pose_small(n_views=2, w=96, h=54, seed=127)
    for P in (-2.0, 0.01):
        with pytest.raises(rvsb.RvsbError) as e:
            gpu_synthesize(ctx, wl.inputs, wl.planes, wl.targets[0], 5.0, params=_params(P))
        assert e.value.status == 7


@pytest.mark.parametrize("case,P,threshold", [(dict(n_views=2, w=128, h=64, seed=128), 2.0, 5000.0),
                                              (dict(n_views=3, w=96, h=54, seed=130), 1.5, 5000.0),
                                              (dict(n_views=2, w=128, h=64, seed=131, erp_in=True), 0.75, 1000.0)],
                         ids=["P2", "P1.5-odd", "P0.75-erp"])
def test_aux_outputs_at_precision(ctx, case, P, threshold):
    """OutputMasks, DepthOutputFiles and MaskedDepthOutputFiles at
    Precision != 1 (Pipeline.cpp:303-333): validity and depth blended at the
    raster size, the mask resized with INTER_NEAREST and the depth with
    INTER_LINEAR to the output size; against the oracle with the tolerances
    of test_gpu_aux.py.  MaskedOutputFiles is refused there: the reference
    masks the raster-sized colour with the output-sized mask, which OpenCV
    rejects."""
    wl = scenes.random_pose_small(**case)
    sc = rvsb.Scene(ctx, wl.inputs)
    for i, p in enumerate(wl.planes):
        sc.upload(i, [np.ascontiguousarray(a, np.uint16) for a in p], on_device=False)
    t = wl.targets[0]
    t.rotation[0] += 3.0
    wo, ho = t.width, t.height
    out = yuv_planes_torch(wo, ho)
    mask = torch.zeros(ho * wo, dtype=torch.uint8, device="cuda")
    depth = torch.zeros(ho * wo, dtype=torch.int16, device="cuda")
    mdepth = torch.zeros(ho * wo, dtype=torch.int16, device="cuda")
    sc.synthesize_aux(t, _params(P), out, mask=mask, depth=depth, masked_depth=mdepth, validity_threshold=threshold)
    torch.cuda.synchronize()
    O.set_precision(P)
    try:
        ref = O.synthesize_aux(wl.inputs, wl.planes, t, 5.0, threshold, masked=False)
    finally:
        O.set_precision(1.0)
    assert_parity(_yuv(out, t), ref["yuv"])
    gmask = mask.cpu().numpy().reshape(ho, wo)
    assert set(np.unique(gmask)) <= {0, 255} and ref["mask"].any() and (~ref["mask"].astype(bool)).any()
    assert (gmask != ref["mask"]).mean() <= 1e-3
    for g, r in ((depth, ref["depth"]), (mdepth, ref["masked_depth"])):
        diff = np.abs(to_u16(g, (ho, wo)).astype(np.int64) - r.astype(np.int64))
        assert (diff > 1).mean() <= 5e-3, f"{(diff > 1).mean():.4f} of depth samples differ by more than 1"
    masked = yuv_planes_torch(wo, ho)
    with pytest.raises(rvsb.RvsbError) as e:
        sc.synthesize_aux(t, _params(P), out, masked=masked)
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
