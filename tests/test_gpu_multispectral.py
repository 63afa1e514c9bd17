"""BlendingMethod Multispectral (BlendedViewMultiSpec): the luma of every
view split by a masked box blur into low and high frequencies, each band
blended with its own factor, the bands added.  The CUDA path against the
oracle's restatement (parity bar of the synthesis)."""
import numpy as np
import pytest

import oracle as O
import rvsb
from rvsb import scenes
from helpers import assert_parity, gpu_synthesize

pytestmark = pytest.mark.gpu

CASES = [
    dict(n_views=3, w=96, h=54, seed=101),
    dict(n_views=2, w=128, h=64, seed=102, erp_in=True),
    dict(n_views=4, w=160, h=96, seed=103),
    dict(n_views=3, w=128, h=64, seed=104, erp_in=True, erp_out=True),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: "-".join(f"{k}{v}" for k, v in c.items()))
@pytest.mark.parametrize("low,high", [(1.0, 8.0), (5.0, 2.0), (-1.0, 4.0)], ids=["1-8", "5-2", "max-4"])
def test_multispectral_matches_oracle(ctx, case, low, high):
    wl = scenes.random_pose_small(**case)
    target = wl.targets[0]
    p = rvsb.params(5.0, multispectral=(low, high))
    yuv, dbg, _ = gpu_synthesize(ctx, wl.inputs, wl.planes, target, 5.0, debug=True, params=p)
    O.set_multispectral(True, low, high)
    try:
        cpu, cq, _ = O.synthesize(wl.inputs, wl.planes, target, 5.0, want_intermediate=True)
    finally:
        O.set_multispectral(False)
    np.testing.assert_array_equal(~(dbg["blend_quality"] > 0), ~(cq > 0))
    assert_parity(yuv, cpu)


def test_multispectral_differs_from_simple(ctx):
    """The mode is really on: the result differs from the simple blend."""
    wl = scenes.random_pose_small(n_views=3, w=96, h=54, seed=105)
    target = wl.targets[0]
    a, _ = gpu_synthesize(ctx, wl.inputs, wl.planes, target, 5.0)
    b, _ = gpu_synthesize(ctx, wl.inputs, wl.planes, target, 5.0, params=rvsb.params(5.0, multispectral=(1.0, 8.0)))
    assert any((x != y).any() for x, y in zip(a, b))
