"""The CUDA path against the committed golden fixtures (tests/golden) and
both output chroma rounding modes of the writer."""
import ctypes
import os

import numpy as np
import pytest

import oracle as O
import rvsb
from rvsb import abi, scenes
from helpers import assert_parity, gpu_synthesize

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _camera(a):
    c = abi.Camera()
    ctypes.memmove(ctypes.addressof(c), a.tobytes(), ctypes.sizeof(c))
    return c


@pytest.mark.parametrize("k", [0, 1, 2])
def test_golden_synthesis(ctx, k):
    z = np.load(os.path.join(GOLDEN, f"synth_small_{k}.npz"))
    n = int(z["n"])
    cams = [_camera(z[f"cam{i}"]) for i in range(n)]
    planes = [(z[f"y{i}"], z[f"u{i}"], z[f"v{i}"], z[f"d{i}"]) for i in range(n)]
    yuv, dbg, _ = gpu_synthesize(ctx, cams, planes, _camera(z["target"]), float(z["exponent"]), debug=True)
    np.testing.assert_array_equal(dbg["blend_quality"] > 0, z["quality"] > 0)
    assert_parity(yuv, (z["Y"], z["U"], z["V"]))


@pytest.mark.parametrize("mode", [rvsb.CHROMA_TIES_EVEN, rvsb.CHROMA_TIES_UP])
def test_chroma_rounding_modes(ctx, mode):
    wl = scenes.random_pose_small(n_views=3, w=96, h=54, seed=41)
    target = wl.targets[0]
    target.rotation[0] += 4.0  # holes, so the inpainting writer is covered too
    yuv, dbg, _ = gpu_synthesize(ctx, wl.inputs, wl.planes, target, 5.0, debug=True,
                                 params=rvsb.params(5.0, chroma_rounding=mode))
    assert (~(dbg["blend_quality"] > 0)).sum() > 0
    O.set_chroma_round(mode)
    try:
        cpu = O.synthesize(wl.inputs, wl.planes, target, 5.0)
    finally:
        O.set_chroma_round(0)
    assert_parity(yuv, cpu)
    # the chroma of each mode is its own rounding of the GPU's Y-resolution
    # codes: recompute it from the other mode's output where they may differ
    other, _, _ = gpu_synthesize(ctx, wl.inputs, wl.planes, target, 5.0, debug=True,
                                 params=rvsb.params(5.0, chroma_rounding=1 - mode))
    for a, b in zip(yuv[1:], other[1:]):
        d = a.astype(np.int32) - b.astype(np.int32)
        assert np.abs(d).max() <= 1
        assert (d != 0).any()


def test_rejects_bad_rounding_mode(ctx):
    wl = scenes.random_pose_small(n_views=1, w=64, h=36, seed=3)
    with pytest.raises(rvsb.RvsbError):
        gpu_synthesize(ctx, wl.inputs, wl.planes, wl.targets[0], 5.0, params=rvsb.params(5.0, chroma_rounding=2))
