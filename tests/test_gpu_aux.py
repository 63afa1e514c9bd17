"""Auxiliary outputs (rvsb_synthesize_aux) against the oracle: the validity
mask, the masked colour, the blended depth and the masked depth of the
reference's CPU mode (Pipeline.cpp:303-336)."""
import numpy as np
import pytest

import oracle as O
import rvsb
from rvsb import scenes
from helpers import assert_parity, to_u16, yuv_planes_torch

pytestmark = pytest.mark.gpu

CASES = [
    dict(n_views=3, w=96, h=54, seed=81),
    dict(n_views=2, w=128, h=64, seed=82, erp_in=True),
    dict(n_views=4, w=80, h=48, seed=83),
    dict(n_views=3, w=128, h=64, seed=84, erp_in=True, erp_out=True),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: "-".join(f"{k}{v}" for k, v in c.items()))
@pytest.mark.parametrize("threshold,exponent", [(5000.0, 5.0), (9000.0, 5.0), (5000.0, -1.0)],
                         ids=["t5000", "t9000", "t5000-by_max"])
def test_aux_outputs_match_oracle(ctx, case, threshold, exponent):
    import torch
    wl = scenes.random_pose_small(**case)
    target = wl.targets[0]
    target.rotation[0] += 3.0
    sc = rvsb.Scene(ctx, wl.inputs)
    for i, p in enumerate(wl.planes):
        sc.upload(i, [np.ascontiguousarray(a, np.uint16) for a in p], on_device=False)
    wo, ho = target.width, target.height
    out = yuv_planes_torch(wo, ho)
    masked = yuv_planes_torch(wo, ho)
    mask = torch.zeros(wo * ho, dtype=torch.uint8, device="cuda")
    depth = torch.zeros(wo * ho, dtype=torch.int16, device="cuda")
    mdepth = torch.zeros(wo * ho, dtype=torch.int16, device="cuda")
    sc.synthesize_aux(target, rvsb.params(exponent), out, mask=mask, masked=masked, depth=depth,
                      masked_depth=mdepth, validity_threshold=threshold)
    torch.cuda.synchronize()
    ref = O.synthesize_aux(wl.inputs, wl.planes, target, exponent, threshold)
    yuv = (to_u16(out[0], (ho, wo)), to_u16(out[1], (ho // 2, wo // 2)), to_u16(out[2], (ho // 2, wo // 2)))
    assert_parity(yuv, ref["yuv"])
    gmask = mask.cpu().numpy().reshape(ho, wo)
    assert set(np.unique(gmask)) <= {0, 255}
    assert (gmask != ref["mask"]).mean() <= 1e-3
    assert ref["mask"].any()
    myuv = (to_u16(masked[0], (ho, wo)), to_u16(masked[1], (ho // 2, wo // 2)),
            to_u16(masked[2], (ho // 2, wo // 2)))
    assert_parity(myuv, ref["masked_yuv"])
    for g, r in ((depth, ref["depth"]), (mdepth, ref["masked_depth"])):
        gd = to_u16(g, (ho, wo)).astype(np.int64)
        diff = np.abs(gd - r.astype(np.int64))
        assert (diff > 1).mean() <= 5e-3, f"{(diff > 1).mean():.4f} of depth samples differ by more than 1"


def test_aux_off_matches_plain(ctx):
    """Asking for no auxiliary output changes nothing in the colour output."""
    import torch
    wl = scenes.random_pose_small(n_views=2, w=96, h=54, seed=85)
    target = wl.targets[0]
    sc = rvsb.Scene(ctx, wl.inputs)
    for i, p in enumerate(wl.planes):
        sc.upload(i, [np.ascontiguousarray(a, np.uint16) for a in p], on_device=False)
    a = yuv_planes_torch(target.width, target.height)
    b = yuv_planes_torch(target.width, target.height)
    sc.synthesize(target, rvsb.params(5.0), a)
    depth = torch.zeros(target.width * target.height, dtype=torch.int16, device="cuda")
    sc.synthesize_aux(target, rvsb.params(5.0), b, depth=depth)
    torch.cuda.synchronize()
    for x, y in zip(a, b):
        assert torch.equal(x, y)
