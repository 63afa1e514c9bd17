"""Batches (rvsb_synthesize_batch): every slot's output is bit-identical to
the per-view call for the same camera, whatever the batch composition
(mixed output sizes and projections, partial groups), with and without
CUDA graphs."""
import copy

import numpy as np
import pytest

import oracle as O
import rvsb
from rvsb import abi, scenes
from helpers import (assert_mask_against_reference, assert_parity, gpu_hole_mask, parallel_map,
                     reference_and_oracle, to_u16, yuv_planes_torch)

pytestmark = pytest.mark.gpu


def _upload(ctx, wl):
    sc = rvsb.Scene(ctx, wl.inputs)
    for i, p in enumerate(wl.planes):
        sc.upload(i, [np.ascontiguousarray(a, np.uint16) for a in p], on_device=False)
    return sc


def _yuv(out, cam):
    wo, ho = cam.width, cam.height
    return (to_u16(out[0], (ho, wo)), to_u16(out[1], (ho // 2, wo // 2)), to_u16(out[2], (ho // 2, wo // 2)))


def _single(sc, cam, p):
    import torch
    out = yuv_planes_torch(cam.width, cam.height)
    sc.synthesize(cam, p, out)
    torch.cuda.synchronize()
    return _yuv(out, cam)


def _targets_small(wl):
    base = wl.targets[0]
    cams = []
    for k in range(5):
        c = copy.deepcopy(base)
        c.position[1] += 0.01 * (k - 2)
        c.rotation[0] += 1.5 * (k - 2)
        if k == 1:  # a smaller output
            c.width, c.height = 64, 36
            c.focal[0] = c.focal[1] = c.focal[0] * 64 / base.width
            c.principle_point[0], c.principle_point[1] = 32.0, 18.0
        if k == 3:  # a 360-degree output
            c = abi.make_camera(abi.EQUIRECTANGULAR, 128, 64, tuple(base.position), (10.0, 0, 0), (0.3, 20.0))
        cams.append(c)
    return cams


@pytest.mark.parametrize("graphs", [False, True])
@pytest.mark.parametrize("slots", [1, 3, 8])
def test_batch_matches_single(ctx, graphs, slots):
    import torch
    wl = scenes.random_pose_small(n_views=3, w=96, h=54, seed=51)
    sc = _upload(ctx, wl)
    cams = _targets_small(wl)
    p = rvsb.params(5.0)
    expected = [_single(sc, c, p) for c in cams]
    b = rvsb.Batch(sc, slots, graphs=graphs)
    for rep in range(2):  # the second pass replays the captured graphs
        outs = [yuv_planes_torch(c.width, c.height) for c in cams]
        b.synthesize(cams, p, outs)
        torch.cuda.synchronize()
        for c, o, e in zip(cams, outs, expected):
            for x, y in zip(_yuv(o, c), e):
                np.testing.assert_array_equal(x, y)
    # 10 launches, plus the two column-group pre-passes of the inpainting
    # when the batch's strips alone do not fill the device
    assert b.last_launch_count() in (10, 12)
    b.close()


def test_batch_matches_oracle(ctx):
    import torch
    wl = scenes.random_pose_small(n_views=2, w=96, h=54, seed=52)
    sc = _upload(ctx, wl)
    cams = _targets_small(wl)[:3]
    outs = [yuv_planes_torch(c.width, c.height) for c in cams]
    b = rvsb.Batch(sc, 4, graphs=True)
    b.synthesize(cams, rvsb.params(5.0), outs)
    torch.cuda.synchronize()
    for c, o in zip(cams, outs):
        assert_parity(_yuv(o, c), O.synthesize(wl.inputs, wl.planes, c, 5.0))


def test_batch_1080p_matches_single(ctx):
    import torch
    wl = scenes.plain_1080p(n_targets=6)
    sc = _upload(ctx, wl)
    p = rvsb.params(wl.blending_factor)
    expected = [_single(sc, c, p) for c in wl.targets]
    b = rvsb.Batch(sc, 4, graphs=True)
    b.reserve(1920, 1080)
    outs = [yuv_planes_torch(c.width, c.height) for c in wl.targets]
    b.synthesize(wl.targets, p, outs)
    torch.cuda.synchronize()
    for c, o, e in zip(wl.targets, outs, expected):
        for x, y in zip(_yuv(o, c), e):
            np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("erp", [False, True], ids=["persp", "erp"])
def test_every_raster_variant_identical(ctx, erp):
    """Every raster variant the autotuner chooses from (tile sizes, view
    groups, stretched-triangle threshold, staging depth) gives the same
    bytes as the default path, for perspective and wrapped 360 outputs."""
    import torch
    wl = scenes.random_pose_small(n_views=3, w=128, h=64, seed=71, erp_in=erp, erp_out=erp)
    sc = _upload(ctx, wl)
    p = rvsb.params(5.0)
    cams = _targets_small(wl)[:4]
    expected = [_single(sc, c, p) for c in cams]
    b = rvsb.Batch(sc, 4)
    for v in range(rvsb.RASTER_VARIANTS):
        b.set_raster_variant(v)
        outs = [yuv_planes_torch(c.width, c.height) for c in cams]
        b.synthesize(cams, p, outs)
        torch.cuda.synchronize()
        assert b.last_raster_variant() == v
        for c, o, e in zip(cams, outs, expected):
            for x, y in zip(_yuv(o, c), e):
                np.testing.assert_array_equal(x, y)
    b.set_raster_variant(-1)
    b.set_autotune(True)
    outs = [yuv_planes_torch(c.width, c.height) for c in cams]
    b.synthesize(cams, p, outs)
    torch.cuda.synchronize()
    assert 0 <= b.last_raster_variant() < rvsb.RASTER_VARIANTS
    for c, o, e in zip(cams, outs, expected):
        for x, y in zip(_yuv(o, c), e):
            np.testing.assert_array_equal(x, y)
    b.close()


def test_default_raster_variant_follows_magnification(ctx):
    """With no variant pinned and the tuner off, an output at the inputs'
    pixels per radian (small or 1920x1080) runs variant 4 (64x32 tiles of
    four views, 1024-thread CTAs), a 3x magnified one variant 7 (the
    medium-triangle path) and a perspective one minified 3x variant 2
    (32x32 tiles, 1024-thread CTAs); each gives the bytes of another
    variant.  A batch of 8 or more unmagnified views runs variant 1."""
    import torch
    wl = scenes.random_pose_small(n_views=2, w=64, h=36, seed=5)
    sc = _upload(ctx, wl)
    p = rvsb.params(5.0)
    same = wl.targets[0]
    big = copy.deepcopy(same)
    big.width, big.height = 192, 108
    for i in range(2):
        big.focal[i] *= 3.0
        big.principle_point[i] *= 3.0
    wide = copy.deepcopy(same)
    wide.width, wide.height = 1920, 1080
    wide.principle_point[0], wide.principle_point[1] = 960.0, 540.0
    small = copy.deepcopy(same)
    small.width, small.height = 22, 12
    for i in range(2):
        small.focal[i] /= 3.0
        small.principle_point[i] /= 3.0
    b = rvsb.Batch(sc, 1)
    for cam, expected_variant in ((same, 4), (big, 7), (wide, 4), (small, 2)):
        out = yuv_planes_torch(cam.width, cam.height)
        b.synthesize([cam], p, [out])
        torch.cuda.synchronize()
        assert b.last_raster_variant() == expected_variant
        got = _yuv(out, cam)
        b.set_raster_variant(3 if expected_variant == 7 else 6)
        out2 = yuv_planes_torch(cam.width, cam.height)
        b.synthesize([cam], p, [out2])
        torch.cuda.synchronize()
        b.set_raster_variant(-1)
        for x, y in zip(got, _yuv(out2, cam)):
            np.testing.assert_array_equal(x, y)
    b.close()
    # A batch of 8 unmagnified views runs variant 1 (two 512-thread CTAs
    # per SM); its outputs are those of the single-view calls.
    b8 = rvsb.Batch(sc, 8)
    outs = [yuv_planes_torch(same.width, same.height) for _ in range(8)]
    b8.synthesize([same] * 8, p, outs)
    torch.cuda.synchronize()
    assert b8.last_raster_variant() == 1
    b1 = rvsb.Batch(sc, 1)
    alone = yuv_planes_torch(same.width, same.height)
    b1.synthesize([same], p, [alone])
    torch.cuda.synchronize()
    for o in outs:
        for x, y in zip(_yuv(o, same), _yuv(alone, same)):
            np.testing.assert_array_equal(x, y)
    b8.close()
    b1.close()


@pytest.mark.parametrize("name,n,picks", [("batched_erp", 32, (0, 4, 9, 13, 18, 22, 27, 31)),
                                          ("batched_mixed", 64, (0, 1, 2, 9, 20, 33, 47, 63))])
def test_batched_configuration_full_size(ctx, name, n, picks):
    """The batched configurations at full size through the tuned batch call,
    one launch group of the configuration's size: 4 ERP 4096x2048 inputs
    seen by 32 1920x1080 views (magnified: the tuner takes the
    medium-triangle variant) and 11 perspective 2048x1088 inputs seen by 64
    views of mixed sizes.  Eight targets of each against the reference's CPU
    output: the parity bar and the hole mask (from the debug call on the
    same scene, whose output equals the batch slot's) as
    assert_mask_against_reference states."""
    import torch
    wl = getattr(scenes, name)(n_targets=n)
    sc = _upload(ctx, wl)
    p = rvsb.params(wl.blending_factor)
    b = rvsb.Batch(sc, n)
    b.set_autotune(True)
    outs = [yuv_planes_torch(c.width, c.height) for c in wl.targets]
    b.synthesize(wl.targets, p, outs)
    torch.cuda.synchronize()
    print(name, "raster variant", b.last_raster_variant())
    gpu = {}
    for k in picks:
        c = wl.targets[k]
        hole, dyuv = gpu_hole_mask(sc, c, p)
        got = _yuv(outs[k], c)
        for x, y in zip(got, dyuv):
            np.testing.assert_array_equal(x, y)
        gpu[k] = (got, hole)
    b.close()
    sc.close()
    refs = parallel_map(lambda k: reference_and_oracle(wl.inputs, wl.planes, wl.targets[k], wl.blending_factor),
                        list(picks))
    sizes = set()
    for k, (ryuv, rq, oq) in zip(picks, refs):
        got, hole = gpu[k]
        diff = assert_mask_against_reference(hole, rq, oq)
        print(k, wl.targets[k].width, "mask pixels off the reference's", diff, assert_parity(got, ryuv))
        sizes.add((wl.targets[k].width, wl.targets[k].height))
    if name == "batched_mixed":
        assert len(sizes) == 3


@pytest.mark.parametrize("scene_name", ["plain_1080p", "batched_erp"])
def test_erp_output_full_size(ctx, scene_name):
    """The serving mix's largest output class, an equirectangular 4096x2048
    view, at full size from the 4 x 1920x1080 scene and from the 4 x ERP
    4096x2048 room: per-view call and a batch slot against the reference's
    CPU output (parity bar; hole mask as assert_mask_against_reference
    states)."""
    import torch
    wl = getattr(scenes, scene_name)()
    base = wl.targets[0]
    cam = abi.make_camera(abi.EQUIRECTANGULAR, 4096, 2048, tuple(base.position),
                          (base.rotation[0] + 20.0, 0.0, 0.0), tuple(base.depth_range))
    sc = _upload(ctx, wl)
    p = rvsb.params(wl.blending_factor)
    single = _single(sc, cam, p)
    hole, dyuv = gpu_hole_mask(sc, cam, p)
    b = rvsb.Batch(sc, 2)
    outs = [yuv_planes_torch(c.width, c.height) for c in (cam, base)]
    b.synthesize([cam, base], p, outs)
    torch.cuda.synchronize()
    for x, y, z in zip(single, dyuv, _yuv(outs[0], cam)):
        np.testing.assert_array_equal(x, y)
        np.testing.assert_array_equal(x, z)
    b.close()
    sc.close()
    ryuv, rq, oq = reference_and_oracle(wl.inputs, wl.planes, cam, wl.blending_factor)
    diff = assert_mask_against_reference(hole, rq, oq)
    print("mask pixels off the reference's", diff, assert_parity(single, ryuv))


def test_batch_slot_seeing_nothing(ctx):
    """A batch whose first slot's camera faces away from the scene (every
    pixel a hole, nothing to inpaint from) beside slots that see it: each
    slot's bytes equal its per-view call."""
    import torch
    wl = scenes.random_pose_small(n_views=2, w=64, h=36, seed=7)
    sc = _upload(ctx, wl)
    p = rvsb.params(5.0)
    away = copy.deepcopy(wl.targets[0])
    away.rotation[0] += 180.0
    cams = [away] + _targets_small(wl)[:3]
    expected = [_single(sc, c, p) for c in cams]
    b = rvsb.Batch(sc, len(cams))
    outs = [yuv_planes_torch(c.width, c.height) for c in cams]
    b.synthesize(cams, p, outs)
    torch.cuda.synchronize()
    for c, o, e in zip(cams, outs, expected):
        for x, y in zip(_yuv(o, c), e):
            np.testing.assert_array_equal(x, y)
    b.close()
