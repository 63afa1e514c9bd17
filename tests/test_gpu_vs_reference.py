"""The CUDA path (the plain per-view call through the C ABI) against the
reference's own CPU synthesis code (oracle/_ref/libref.so: transform.cpp,
BlendedView.cpp/blending.cpp, inpainting.cpp, image_writing.cpp and the
camera classes, compiled unmodified), without the oracle in between.

Bar: identical hole mask (pre-inpainting !(quality > 0)), Y/U/V PSNR >= 50
dB, <= 0.5% of samples more than 2 codes off; with an equirectangular camera
the mask is identical to the oracle's correctly rounded trigonometry and
within helpers.ERP_MASK_TOLERANCE of the reference's libm result.  The decoded inputs come from
the oracle's loader, which test_gpu_reference_loader.py checks bit for bit
against the reference's loader kernels.
"""
import numpy as np
import pytest

import ref
from rvsb import scenes
from helpers import assert_mask_against_reference, assert_parity, gpu_synthesize, reference_and_oracle

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref.available(), reason="reference harness not built")]

CASES = [
    dict(n_views=2, w=64, h=36, seed=1),
    dict(n_views=3, w=96, h=54, seed=2),
    dict(n_views=4, w=80, h=48, seed=3),
    dict(n_views=2, w=128, h=64, seed=4, erp_in=True),
    dict(n_views=3, w=128, h=64, seed=5, erp_in=True, erp_out=True),
    dict(n_views=2, w=100, h=50, seed=7),
]


def _check(ctx, wl, target, exponent):
    yuv, dbg, _ = gpu_synthesize(ctx, wl.inputs, wl.planes, target, exponent, debug=True)
    plain, _ = gpu_synthesize(ctx, wl.inputs, wl.planes, target, exponent)
    for a, b in zip(plain, yuv):
        np.testing.assert_array_equal(a, b)
    ryuv, rq, oq = reference_and_oracle(wl.inputs, wl.planes, target, exponent)
    assert_mask_against_reference(~(dbg["blend_quality"] > 0), rq, oq)
    return assert_parity(plain, ryuv)


@pytest.mark.parametrize("exponent", [5.0, 1.0, -1.0], ids=["exp5", "exp1", "by_max"])
@pytest.mark.parametrize("case", CASES, ids=lambda c: "-".join(f"{k}{v}" for k, v in c.items()))
def test_small_matches_reference(ctx, case, exponent):
    wl = scenes.random_pose_small(**case)
    _check(ctx, wl, wl.targets[0], exponent)


def test_plain_small_matches_reference(ctx):
    """2 x 960x540 -> 960x540, full size."""
    wl = scenes.plain_small()
    print(_check(ctx, wl, wl.targets[0], 5.0))


def test_plain_1080p_matches_reference(ctx):
    """4 x 1920x1080 -> 1920x1080 (the measured workload), full size."""
    wl = scenes.plain_1080p()
    print(_check(ctx, wl, wl.targets[0], 5.0))
