"""'Precision' (oversampled rasterisation) in the oracle: the output resize
is OpenCV's INTER_LINEAR resize of a float image (write_color,
image_writing.cpp:188-190), checked against OpenCV itself; and the
synthesis at P != 1 against the same synthesis at P = 1."""
import os

import numpy as np
import pytest

import oracle as O
from rvsb import scenes
from helpers import psnr

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

SIZES = [(192, 108, 96, 54), (144, 96, 96, 64), (64, 32, 128, 64), (96, 48, 128, 64), (200, 100, 128, 64),
         (100, 60, 128, 64), (384, 216, 192, 108), (128, 64, 128, 64)]


@pytest.mark.parametrize("ws,hs,wd,hd", SIZES)
def test_resize_matches_opencv(ws, hs, wd, hd):
    """Bit-exact against cv2.resize with OpenCV's optimised (IPP / SIMD)
    paths off, within 2 ulp of the optimised build."""
    cv2 = pytest.importorskip("cv2")
    rng = np.random.default_rng(ws * 1000 + hd)
    img = rng.random((hs, ws, 3), dtype=np.float32)
    ours = O.resize_linear3(img, wd, hd)
    was = cv2.useOptimized()
    try:
        cv2.setUseOptimized(False)
        plain = cv2.resize(img, (wd, hd))
    finally:
        cv2.setUseOptimized(was)
    np.testing.assert_array_equal(ours, plain)
    fast = cv2.resize(img, (wd, hd))
    assert np.abs(ours - fast).max() <= 2.5e-7


def test_resize_exact_2x_is_area_mean():
    img = np.arange(4 * 6 * 3, dtype=np.float32).reshape(4, 6, 3) / 100
    out = O.resize_linear3(img, 3, 2)
    want = ((img[0::2, 0::2] + img[0::2, 1::2]) + (img[1::2, 0::2]) + img[1::2, 1::2]) * np.float32(0.25)
    np.testing.assert_array_equal(out, want.astype(np.float32))


def test_raster_size():
    try:
        O.set_precision(1.5)
        assert O.raster_size(128, 64) == (192, 96)
        assert O.raster_size(96, 54) == (144, 81)
        O.set_precision(0.5)
        assert O.raster_size(96, 54) == (48, 27)
    finally:
        O.set_precision(1.0)
    assert O.raster_size(96, 54) == (96, 54)


@pytest.mark.parametrize("P", [2.0, 1.5, 0.75])
def test_synthesis_close_to_precision_one(P):
    """Oversampling changes the result only at edges: the output stays close
    to the P = 1 synthesis, and differs from it."""
    wl = scenes.random_pose_small(n_views=2, w=128, h=64, seed=111)
    t = wl.targets[0]
    base = O.synthesize(wl.inputs, wl.planes, t, 5.0)
    try:
        O.set_precision(P)
        yuv, q, c = O.synthesize(wl.inputs, wl.planes, t, 5.0, want_intermediate=True)
    finally:
        O.set_precision(1.0)
    assert q.shape == (int(0.5 + 64 * P), int(0.5 + 128 * P))
    assert any((a != b).any() for a, b in zip(yuv, base))
    assert psnr(yuv[0], base[0]) > 25.0


def test_nearest_resize_matches_cv2():
    """The validity mask's resize at Precision != 1 (cv::resize with
    INTER_NEAREST, Pipeline.cpp:303-308) against cv2, from the raster sizes
    of P = 2, 1.5, 0.75, 0.9, 0.5 and 0.7 (odd sides included)."""
    z = np.load(os.path.join(GOLDEN, "cv2_resize_nearest.npz"))
    for k in range(int(z["n"])):
        src, expected = z[f"in{k}"], z[f"out{k}"]
        h, w = expected.shape
        np.testing.assert_array_equal(O.resize_nearest_u8(src, w, h), expected)
