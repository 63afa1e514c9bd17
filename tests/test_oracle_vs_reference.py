"""The CPU oracle against the reference's own code.

oracle/_ref/libref.so is the reference's CPU synthesis path (rvs/src:
Parameters, the (Un)Projectors, SpaceTransformer, transform.cpp,
BlendedView/blending.cpp, View/inpainting.cpp, image_writing.cpp) compiled
unmodified against an OpenCV stand-in (oracle/ref/).  Every stage the oracle
restates is compared with it bit for bit on the seeded small workloads the
GPU parity tests use: relative pose, warped (u, v) and depth, per-view
raster (colour, depth, validity, quality), the blend (simple at exponents 5
and 1, by maximum, multispectral), inpainting (colour and source pixel),
the YUV420 writer and the whole synthesis, plus the committed golden
fixtures.  The GPU path is tested against the oracle, so these tests carry
the GPU's parity through to the reference.

Trigonometry: the reference calls float std::cos/sin/atan2/asin, which this
build takes from the host libm; the oracle matches them bit for bit in its
libm mode (set_trig_mode(1)).  The GPU evaluates them correctly rounded (the
oracle's default mode), and test_erp_correctly_rounded_trig_within_bar
measures that difference against the reference.
"""
import copy
import os

import numpy as np
import pytest

import oracle as O
import ref
from rvsb import abi, scenes
from helpers import parity_report

pytestmark = pytest.mark.skipif(not ref.available(), reason="reference harness not built and reference tree absent")

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

CASES = [
    dict(n_views=2, w=64, h=36, seed=1),
    dict(n_views=3, w=96, h=54, seed=2),
    dict(n_views=4, w=80, h=48, seed=3),
    dict(n_views=2, w=128, h=64, seed=4, erp_in=True),
    dict(n_views=3, w=128, h=64, seed=5, erp_in=True, erp_out=True),
    dict(n_views=1, w=64, h=36, seed=6),
    dict(n_views=2, w=100, h=50, seed=7),
]
IDS = ["-".join(f"{k}{v}" for k, v in c.items()) for c in CASES]


@pytest.fixture
def libm_trig():
    """The oracle's trigonometry as the reference build's (host libm)."""
    O.set_trig_mode(1)
    yield
    O.set_trig_mode(0)


def _eq(a, b):
    np.testing.assert_array_equal(a, b)


def _decoded(wl):
    cols = [O.decode_color(y, u, v, c.bit_depth_color) for c, (y, u, v, d) in zip(wl.inputs, wl.planes)]
    deps = [O.decode_depth(d, c) for c, (y, u, v, d) in zip(wl.inputs, wl.planes)]
    return cols, deps


def _check_stages(wl, target, exponent):
    cols, deps = _decoded(wl)
    views = []
    for cam, col, dep in zip(wl.inputs, cols, deps):
        R1, t1 = ref.relative_pose(cam, target)
        R2, t2 = O.relative_pose(cam, target)
        _eq(R1, R2)
        _eq(t1, t2)
        ruv, rvd, rwrap = ref.warp(cam, target, dep)
        ouv, ovd, owrap = O.warp(cam, target, dep)
        _eq(ruv, ouv)
        _eq(rvd, ovd)
        assert rwrap == owrap
        rc, rd, rq, rv = ref.raster(col, rvd, ruv, target.width, target.height, rwrap)
        oc, od, ov = O.raster(col, ovd, ouv, target.width, target.height, owrap)
        _eq(rc, oc)
        _eq(rd, od)
        _eq(rv, ov)
        with np.errstate(invalid="ignore", divide="ignore"):
            _eq(rq, ov / od)
        views.append((rc, rd, rq, rv))
    bc, bq, _, _ = ref.blend(*[[v[k] for v in views] for k in range(4)], exponent)
    oc, oq = O.blend([v[0] for v in views], [v[2] for v in views], [v[1] for v in views], exponent)
    _eq(bc, oc)
    _eq(bq, oq)
    hole = ~(bq > 0)
    ri = ref.inpaint(bc, bq)
    oi, osrc, _ = O.inpaint(bc, bq)
    _eq(ri, oi)
    _eq(ref.inpaint_sources(hole)[hole], osrc[hole])
    for a, b in zip(ref.write_color(ri, target), O.write_yuv420(oi, target.bit_depth_color)):
        _eq(a, b)
    # the whole synthesis, loaders aside
    sc, sq = ref.synthesize(wl.inputs, cols, deps, target, exponent)
    yuv, q, _ = O.synthesize(wl.inputs, wl.planes, target, exponent, want_intermediate=True)
    _eq(sq, q)
    for a, b in zip(ref.write_color(sc, target), yuv):
        _eq(a, b)
    return hole


@pytest.mark.parametrize("exponent", [5.0, 1.0, -1.0], ids=["exp5", "exp1", "by_max"])
@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_stages_match_reference(case, exponent, libm_trig):
    wl = scenes.random_pose_small(**case)
    hole = _check_stages(wl, wl.targets[0], exponent)
    assert hole.size > 0


@pytest.mark.parametrize("case", [c for c in CASES if c.get("erp_in")], ids=[i for c, i in zip(CASES, IDS)
                                                                             if c.get("erp_in")])
def test_erp_correctly_rounded_trig_within_bar(case):
    """The oracle's default (and the GPU's) trigonometry, correctly rounded
    float results, against the reference's libm calls: identical hole mask,
    output within the parity bar."""
    wl = scenes.random_pose_small(**case)
    target = wl.targets[0]
    cols, deps = _decoded(wl)
    sc, sq = ref.synthesize(wl.inputs, cols, deps, target, 5.0)
    yuv, q, _ = O.synthesize(wl.inputs, wl.planes, target, 5.0, want_intermediate=True)
    _eq(sq > 0, q > 0)
    r = parity_report(yuv, ref.write_color(sc, target))
    assert min(r["psnr_Y"], r["psnr_U"], r["psnr_V"]) >= 50.0 and r["frac_gt2"] == 0.0, r


@pytest.mark.parametrize("low,high", [(1.0, 8.0), (5.0, 2.0), (-1.0, 4.0)])
@pytest.mark.parametrize("seed", [2, 3])
def test_multispectral_matches_reference(seed, low, high):
    """BlendedViewMultiSpec (BlendedView.cpp:63-88, blending.cpp:62-159,
    371-395): the band split with the integral-image box blur, both bands
    blended with their own factors."""
    wl = scenes.random_pose_small(n_views=3, w=96, h=54, seed=seed)
    target = wl.targets[0]
    cols, deps = _decoded(wl)
    O.set_multispectral(True, low, high)
    try:
        sc, sq = ref.synthesize(wl.inputs, cols, deps, target, 0.0, multispectral=(low, high))
        yuv, q, _ = O.synthesize(wl.inputs, wl.planes, target, 0.0, want_intermediate=True)
    finally:
        O.set_multispectral(False)
    _eq(sq, q)
    for a, b in zip(ref.write_color(sc, target), yuv):
        _eq(a, b)


@pytest.mark.parametrize("precision", [2.0, 1.5, 0.75, 0.5])
def test_precision_raster_matches_reference(precision):
    """'Precision' (g_rescale): the raster at int(0.5 + W * P) with scaled
    uv and the quality stretch divided by P; blended quality and the
    inpainted colour at the raster size (the final resize is OpenCV's,
    pinned against cv2 by test_oracle_precision.py)."""
    wl = scenes.random_pose_small(n_views=2, w=64, h=36, seed=11)
    target = wl.targets[0]
    cols, deps = _decoded(wl)
    O.set_precision(precision)
    ref.set_raster_precision(precision)
    try:
        sc, sq = ref.synthesize(wl.inputs, cols, deps, target, 5.0)
        _, q, c = O.synthesize(wl.inputs, wl.planes, target, 5.0, want_intermediate=True)
    finally:
        O.set_precision(1.0)
        ref.set_raster_precision(1.0)
    _eq(sq, q)
    oi, _, _ = O.inpaint(c, q)
    _eq(sc, oi)


def test_view_facing_away_matches_reference():
    """No input pixel lands in the view: every pixel a hole, no inpainting
    source, the empty colour written."""
    wl = scenes.random_pose_small(n_views=2, w=64, h=36, seed=7)
    target = copy.deepcopy(wl.targets[0])
    target.rotation[0] += 180.0
    hole = _check_stages(wl, target, 5.0)
    assert hole.all()


def _camera(raw):
    return abi.Camera.from_buffer_copy(bytes(raw))


@pytest.mark.parametrize("k", [0, 1, 2])
def test_golden_fixtures_match_reference(k):
    """The committed oracle fixtures (tests/golden/synth_small_*) against the
    reference: bit-exact for the perspective cases; the ERP case was
    recorded with correctly rounded trigonometry, so there the hole mask is
    identical and the output within the parity bar."""
    z = np.load(os.path.join(GOLDEN, f"synth_small_{k}.npz"))
    n = int(z["n"])
    inputs = [_camera(z[f"cam{i}"]) for i in range(n)]
    target = _camera(z["target"])
    cols = [O.decode_color(z[f"y{i}"], z[f"u{i}"], z[f"v{i}"], inputs[i].bit_depth_color) for i in range(n)]
    deps = [O.decode_depth(z[f"d{i}"], inputs[i]) for i in range(n)]
    sc, sq = ref.synthesize(inputs, cols, deps, target, float(z["exponent"]))
    yuv = ref.write_color(sc, target)
    expected = (z["Y"], z["U"], z["V"])
    erp = any(c.projection == abi.EQUIRECTANGULAR for c in inputs + [target])
    _eq(sq > 0, z["quality"] > 0)
    if erp:
        r = parity_report(yuv, expected)
        assert min(r["psnr_Y"], r["psnr_U"], r["psnr_V"]) >= 50.0 and r["frac_gt2"] == 0.0, r
    else:
        _eq(sq, z["quality"])
        for a, b in zip(yuv, expected):
            _eq(a, b)


@pytest.mark.parametrize("ties_up", [0, 1], ids=["ipp", "noipp"])
def test_reference_writer_chroma_matches_cv2(ties_up):
    """The stand-in's cv::resize(0.5, 0.5, INTER_LINEAR) as the reference's
    writer runs it, against the cv2 fixture (both OpenCV builds)."""
    z = np.load(os.path.join(GOLDEN, "cv2_resize_half.npz"))
    suffix = "_noipp" if ties_up else ""
    ref.set_resize_ties_up(ties_up)
    try:
        for k in range(int(z["n"])):
            codes, expected = z[f"in{k}"], z[f"out{k}{suffix}"]
            h, w = codes.shape
            color = np.zeros((h, w, 3), np.float32)
            color[..., 1] = ((codes.astype(np.float64) + 0.5) / 1023.0).astype(np.float32)
            _, U, _ = ref.write_color(color, abi.make_camera(abi.PERSPECTIVE, w, h))
            _eq(U, expected)
    finally:
        ref.set_resize_ties_up(0)


def test_reference_padded_aux_outputs_are_zero():
    """The reference's depth and mask writers with a virtual Crop_region
    (image_writing.cpp:262-267, 285-290) pad with `padded(region) = image`,
    an OpenCV header assignment that copies no data: the file's luma is all
    zero at the padded resolution.  Without a crop the image itself is
    written.  The CLI reproduces both (test_gpu_cli.py)."""
    cam = abi.make_camera(abi.PERSPECTIVE, 32, 16)
    depth = np.linspace(1.0, 5.0, 32 * 16, dtype=np.float32).reshape(16, 32)
    mask = np.zeros((16, 32), np.uint8)
    mask[3:5, 4:9] = 1
    plain = ref.write_aux("depth", depth, None, cam)
    assert plain.shape == (16, 32) and plain.min() > 0
    m = ref.write_aux("mask", None, mask, cam)
    np.testing.assert_array_equal(m, mask * 255)
    crop, padded = (8, 4, 32, 16), (64, 32)
    assert not ref.write_aux("depth", depth, None, cam, crop, padded).any()
    assert not ref.write_aux("masked_depth", depth, mask, cam, crop, padded).any()
    assert not ref.write_aux("mask", None, mask, cam, crop, padded).any()
