"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Bar (per the synthesis spec): Y/U/V PSNR >= 50 dB against the oracle's
output, <= 0.5% of samples differing by more than 2 codes, and an identical
hole mask.  Stage checks are stricter: warped (u, v, depth) are bit-exact,
per-view coverage and the hole mask are identical, and inpainting copies the
same source pixel.
"""
import numpy as np
import pytest

import oracle as O
import rvsb
from rvsb import scenes
from helpers import assert_parity, gpu_synthesize, parity_report

pytestmark = pytest.mark.gpu

SMALL_CASES = [
    dict(n_views=2, w=64, h=36, seed=1),
    dict(n_views=3, w=96, h=54, seed=2),
    dict(n_views=4, w=80, h=48, seed=3),
    dict(n_views=2, w=128, h=64, seed=4, erp_in=True),
    dict(n_views=3, w=128, h=64, seed=5, erp_in=True, erp_out=True),
    dict(n_views=1, w=64, h=36, seed=6),
    dict(n_views=2, w=100, h=50, seed=7),  # width not a multiple of 8: the 2x2 colour decode
]


def _oracle_stages(wl, target, exponent):
    """CPU oracle stage by stage: warped uv/z, per-view raster, blend."""
    warped, views = [], []
    for cam, (y, u, v, d) in zip(wl.inputs, wl.planes):
        col = O.decode_color(y, u, v, cam.bit_depth_color)
        dep = O.decode_depth(d, cam)
        uv, vd, wrap = O.warp(cam, target, dep)
        warped.append((uv, vd))
        oc, od, ov = O.raster(col, vd, uv, target.width, target.height, wrap)
        views.append((oc, od, ov))
    qual = [ov / od for (oc, od, ov) in views]
    bc, bq = O.blend([v[0] for v in views], qual, [v[1] for v in views], exponent)
    return warped, views, bc, bq


@pytest.mark.parametrize("case", SMALL_CASES, ids=lambda c: "-".join(f"{k}{v}" for k, v in c.items()))
@pytest.mark.parametrize("exponent", [5.0, 1.0, -1.0], ids=["exp5", "exp1", "by_max"])
def test_stages_small(ctx, case, exponent):
    wl = scenes.random_pose_small(**case)
    target = wl.targets[0]
    yuv, dbg, _ = gpu_synthesize(ctx, wl.inputs, wl.planes, target, exponent, debug=True)
    warped, views, bc, bq = _oracle_stages(wl, target, exponent)
    # 1. warp: bit-exact (NaN where the CPU writes NaN)
    for v, (uv, vd) in enumerate(warped):
        g = dbg["warped"][v]
        np.testing.assert_array_equal(g[..., 0], uv[..., 0])
        np.testing.assert_array_equal(g[..., 1], uv[..., 1])
        np.testing.assert_array_equal(g[..., 2], vd)
    # 2. raster: identical coverage, same winner colour/depth
    for v, (oc, od, ov) in enumerate(views):
        gcov = dbg["view_validity"][v] > 0
        ccov = ov > 0
        assert np.array_equal(gcov, ccov), f"view {v}: coverage differs at {np.argwhere(gcov != ccov)[:5]}"
        same = np.isclose(dbg["view_depth"][v], od, rtol=1e-5) | (~ccov)
        assert same.mean() > 0.995
        np.testing.assert_allclose(dbg["view_color"][v][ccov], oc[ccov], atol=2e-3)
    # 3. blend: identical hole mask, close colour
    ghole = ~(dbg["blend_quality"] > 0)
    chole = ~(bq > 0)
    assert np.array_equal(ghole, chole)
    np.testing.assert_allclose(dbg["blend_color"], bc, atol=2e-3)
    # 4. end to end
    cpu = O.synthesize(wl.inputs, wl.planes, target, exponent)
    assert_parity(yuv, cpu)


@pytest.mark.parametrize("bits,far,invalid", [(10, 10.0, True), (12, 10.0, False), (16, 2000.0, True)],
                         ids=["10bit", "12bit-valid", "16bit-far-infinite"])
def test_depth_formats(ctx, bits, far, invalid):
    """Depth decode through the per-view table of all 65536 samples:
    bit depths below 16, HasInvalidDepth off, and Depth_range far >= 1000
    (near / d), each bit-exact in the warped vertices and at parity end to
    end."""
    wl = scenes.random_pose_small(n_views=3, w=96, h=54, seed=21)
    for c in wl.inputs:
        c.bit_depth_depth = bits
        c.depth_range[1] = far
        c.has_invalid_depth = 1 if invalid else 0
    target = wl.targets[0]
    yuv, dbg, _ = gpu_synthesize(ctx, wl.inputs, wl.planes, target, 5.0, debug=True)
    warped, _, _, bq = _oracle_stages(wl, target, 5.0)
    for v, (uv, vd) in enumerate(warped):
        g = dbg["warped"][v]
        np.testing.assert_array_equal(g[..., 0], uv[..., 0])
        np.testing.assert_array_equal(g[..., 1], uv[..., 1])
        np.testing.assert_array_equal(g[..., 2], vd)
    np.testing.assert_array_equal(~(dbg["blend_quality"] > 0), ~(bq > 0))
    assert_parity(yuv, O.synthesize(wl.inputs, wl.planes, target, 5.0))


@pytest.mark.parametrize("seed,yaw", [(31, 0.0), (32, 100.0), (33, -150.0)])
def test_erp_tile_culling(ctx, seed, yaw):
    """ERP inputs seen by a perspective output: vertex tiles wholly beyond a
    side of the output are skipped (no triangle from them can cover a
    pixel).  The output, with culling, against the oracle, which warps every
    vertex; and against the GPU's own result with culling off (the debug
    call, which returns the warped vertices, warps every vertex), bit for
    bit."""
    import copy
    wl = scenes.random_pose_small(n_views=2, w=512, h=256, seed=seed, erp_in=True)
    target = copy.deepcopy(wl.targets[0])
    target.rotation[0] = yaw
    yuv, _ = gpu_synthesize(ctx, wl.inputs, wl.planes, target, 5.0)
    full, _, _ = gpu_synthesize(ctx, wl.inputs, wl.planes, target, 5.0, debug=True)
    for a, b in zip(yuv, full):
        np.testing.assert_array_equal(a, b)
    assert_parity(yuv, O.synthesize(wl.inputs, wl.planes, target, 5.0))


@pytest.mark.parametrize("seed", [11, 12, 13])
def test_inpaint_sources_match(ctx, seed):
    """Holes copy exactly the pixel the reference's sweeps choose."""
    wl = scenes.random_pose_small(n_views=2, w=96, h=54, seed=seed)
    target = wl.targets[0]
    target.rotation[0] += 6.0  # rotate away to open border holes
    yuv, dbg, _ = gpu_synthesize(ctx, wl.inputs, wl.planes, target, 5.0, debug=True)
    q = dbg["blend_quality"]
    hole = ~(q > 0)
    assert hole.sum() > 20
    _, src, _ = O.inpaint(dbg["blend_color"], q)
    np.testing.assert_array_equal(dbg["inpaint_source"][hole], src[hole])


def test_deterministic(ctx):
    wl = scenes.random_pose_small(n_views=3, w=96, h=54, seed=21)
    a, _ = gpu_synthesize(ctx, wl.inputs, wl.planes, wl.targets[0], 5.0)
    b, _ = gpu_synthesize(ctx, wl.inputs, wl.planes, wl.targets[0], 5.0)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


def test_plain_small_full_size(ctx):
    """2 x 960x540 -> 960x540 (the CPU-runnable workload), full size."""
    wl = scenes.plain_small()
    target = wl.targets[0]
    yuv, dbg, _ = gpu_synthesize(ctx, wl.inputs, wl.planes, target, 5.0, debug=True)
    cpu, cq, _ = O.synthesize(wl.inputs, wl.planes, target, 5.0, want_intermediate=True)
    assert np.array_equal(~(dbg["blend_quality"] > 0), ~(cq > 0))
    r = assert_parity(yuv, cpu)
    print(r)


def test_plain_1080p_full_size(ctx):
    """4 x 1920x1080 -> 1920x1080 (the headline workload), full size."""
    wl = scenes.plain_1080p()
    target = wl.targets[0]
    yuv, dbg, _ = gpu_synthesize(ctx, wl.inputs, wl.planes, target, 5.0, debug=True)
    cpu, cq, _ = O.synthesize(wl.inputs, wl.planes, target, 5.0, want_intermediate=True)
    assert np.array_equal(~(dbg["blend_quality"] > 0), ~(cq > 0))
    r = assert_parity(yuv, cpu)
    print(r)


def test_frame_call_matches_scene_call(ctx):
    """rvsb_synthesize_frame (device planes, no copies) gives the same bytes
    as rvsb_scene_upload + rvsb_synthesize."""
    import torch
    from helpers import to_u16, yuv_planes_torch
    wl = scenes.random_pose_small(n_views=3, w=96, h=54, seed=31)
    target = wl.targets[0]
    a, sc = gpu_synthesize(ctx, wl.inputs, wl.planes, target, 5.0)
    dev = [[torch.from_numpy(np.ascontiguousarray(x).view(np.int16)).reshape(-1).cuda() for x in pl]
           for pl in wl.planes]
    out = yuv_planes_torch(target.width, target.height)
    sc2 = rvsb.Scene(ctx, wl.inputs)
    sc2.synthesize_frame(dev, target, rvsb.params(5.0), out)
    torch.cuda.synchronize()
    wo, ho = target.width, target.height
    b = (to_u16(out[0], (ho, wo)), to_u16(out[1], (ho // 2, wo // 2)), to_u16(out[2], (ho // 2, wo // 2)))
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("seed,mag", [(41, 4), (42, 6)])
def test_magnified_every_raster_variant(ctx, seed, mag):
    """Low-resolution inputs seen 4x or 6x magnified: most triangles'
    candidate boxes hold 9 to 49 pixels, across the 5 to 32 range that the
    medium-triangle path of raster variants 6 and 7 rasterises with one lane
    per candidate pixel, and above it.  Every variant of the per-view call
    against the oracle, and bit for bit against the default variant."""
    import copy
    import torch
    wl = scenes.random_pose_small(n_views=2, w=48, h=28, seed=seed)
    target = copy.deepcopy(wl.targets[0])
    target.width, target.height = 48 * mag, 28 * mag
    for i in range(2):
        target.focal[i] *= mag
        target.principle_point[i] *= mag
    sc = rvsb.Scene(ctx, wl.inputs)
    for i, p in enumerate(wl.planes):
        sc.upload(i, [np.ascontiguousarray(a, np.uint16) for a in p], on_device=False)
    results = []
    for v in list(range(rvsb.RASTER_VARIANTS)) + [-1]:
        sc.set_raster_variant(v)
        yuv, _ = gpu_synthesize(ctx, wl.inputs, wl.planes, target, 5.0, scene=sc)
        results.append(yuv)
    torch.cuda.synchronize()
    assert_parity(results[0], O.synthesize(wl.inputs, wl.planes, target, 5.0))
    for yuv in results[1:]:
        for a, b in zip(yuv, results[0]):
            np.testing.assert_array_equal(a, b)


def test_view_facing_away(ctx):
    """A virtual camera that sees none of the scene: every pixel is a hole
    and there is no source to inpaint from, so the output is the empty
    colour (0, 1, 0) quantised, as the oracle's, with the whole frame in the
    hole mask; the plain call and the debug call alike."""
    import copy
    wl = scenes.random_pose_small(n_views=2, w=64, h=36, seed=7)
    target = copy.deepcopy(wl.targets[0])
    target.rotation[0] += 180.0
    cpu, cq, _ = O.synthesize(wl.inputs, wl.planes, target, 5.0, want_intermediate=True)
    assert not (cq > 0).any()
    plain, _ = gpu_synthesize(ctx, wl.inputs, wl.planes, target, 5.0)
    dyuv, dbg, _ = gpu_synthesize(ctx, wl.inputs, wl.planes, target, 5.0, debug=True)
    assert not (dbg["blend_quality"] > 0).any()
    for yuv in (plain, dyuv):
        for a, b in zip(yuv, cpu):
            np.testing.assert_array_equal(a, b)
