"""rvsb_inpaint_sources_noalloc (static device scratch, no allocation)
against the inpainting sources the regular synthesis entry point reports
(rvsb_synthesize_debug), on two calls in a row.  Integer sources: the bar is
exact equality.  This file sorts last so the entry point also runs after
every other test in the same process."""
import numpy as np
import pytest

import oracle as O
import rvsb
from rvsb import scenes
from helpers import gpu_synthesize
from inpaint_model import inpaint_sources

pytestmark = pytest.mark.gpu

MAX_PIXELS = 1 << 19


def _holes_and_sources(ctx, wl, target):
    _, dbg, _ = gpu_synthesize(ctx, wl.inputs, wl.planes, target, 5.0, debug=True)
    hole = ~(dbg["blend_quality"] > 0)
    return hole, dbg["inpaint_source"]


def _noalloc(hole):
    import torch
    h, w = hole.shape
    dev_holes = torch.from_numpy(hole.astype(np.uint8)).cuda()
    out = []
    for _ in range(2):  # two calls in a row on the same scratch
        src = torch.full((h, w, 2), -7, dtype=torch.int32, device="cuda")
        rvsb.inpaint_sources_noalloc(dev_holes, w, h, src)
        torch.cuda.synchronize()
        out.append(src.cpu().numpy())
    return out


def _check(hole, expected, got):
    h, w = hole.shape
    ys, xs = np.mgrid[0:h, 0:w]
    for s in got:
        np.testing.assert_array_equal(s[hole], expected[hole])
        np.testing.assert_array_equal(s[~hole][:, 0], xs[~hole])
        np.testing.assert_array_equal(s[~hole][:, 1], ys[~hole])


@pytest.mark.parametrize("seed", [11, 12])
def test_noalloc_matches_synthesis_small(ctx, seed):
    wl = scenes.random_pose_small(n_views=2, w=96, h=54, seed=seed)
    target = wl.targets[0]
    target.rotation[0] += 6.0  # rotate away to open border holes
    hole, expected = _holes_and_sources(ctx, wl, target)
    _check(hole, expected, _noalloc(hole))


def test_noalloc_matches_synthesis_960x540(ctx):
    """The 2 x 960x540 workload with the target turned to open holes: the
    largest standard size within the scratch limit."""
    wl = scenes.plain_small()
    target = wl.targets[0]
    target.rotation[0] += 3.0
    assert target.width * target.height <= MAX_PIXELS
    hole, expected = _holes_and_sources(ctx, wl, target)
    _check(hole, expected, _noalloc(hole))


def test_noalloc_rejects_oversize():
    import torch
    w, h = 1024, 1024
    holes = torch.zeros(w * h, dtype=torch.uint8, device="cuda")
    src = torch.zeros(w * h * 2, dtype=torch.int32, device="cuda")
    with pytest.raises(rvsb.RvsbError) as e:
        rvsb.inpaint_sources_noalloc(holes, w, h, src)
    assert "exceeds the no-allocation scratch limit" in str(e.value)


def _oracle_sources(hole):
    h, w = hole.shape
    q = np.where(hole, 0.0, 1.0).astype(np.float32)
    _, src, _ = O.inpaint(np.zeros((h, w, 3), np.float32), q)
    return src


@pytest.mark.parametrize("kind", ["all_holes", "no_holes", "one_source"])
def test_noalloc_degenerate_masks(kind):
    """Masks the synthesis tests reach only through whole scenes: every
    pixel a hole (no source exists, so every pixel reports itself, as the
    reference's map starts and stays), no hole at all, and a single
    non-hole pixel that every hole takes.  Checked against the oracle's
    literal sweeps and the numpy scan model."""
    h, w = 36, 64
    hole = np.ones((h, w), bool) if kind != "no_holes" else np.zeros((h, w), bool)
    if kind == "one_source":
        hole[20, 41] = False
    expected = _oracle_sources(hole)
    np.testing.assert_array_equal(inpaint_sources(hole)[hole], expected[hole])
    _check(hole, expected, _noalloc(hole))
