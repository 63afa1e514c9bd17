"""Shared test helpers: run the CUDA path through the C ABI and compare it
with the CPU oracle."""
import numpy as np

import oracle as O
import rvsb


def yuv_planes_torch(wo, ho):
    import torch
    return [torch.empty(n, dtype=torch.int16, device="cuda")
            for n in (wo * ho, (wo // 2) * (ho // 2), (wo // 2) * (ho // 2))]


def to_u16(t, shape):
    return t.cpu().numpy().view(np.uint16).reshape(shape)


def gpu_synthesize(ctx, inputs, planes, target, exponent, debug=False, scene=None, params=None):
    """Synthesises `target` on the GPU.  Returns (Y, U, V) uint16 arrays and,
    with debug=True, a dict of intermediate results."""
    import torch
    sc = scene or rvsb.Scene(ctx, inputs)
    if scene is None:
        for i, p in enumerate(planes):
            sc.upload(i, [np.ascontiguousarray(a, np.uint16) for a in p], on_device=False)
    wo, ho = target.width, target.height
    out = yuv_planes_torch(wo, ho)
    p = params if params is not None else rvsb.params(exponent)
    dbg = None
    if debug:
        # intermediates are at the raster size (Precision P: int(0.5 + W * P))
        ow, oh = wo, ho
        if p.precision != 1.0:
            P = np.float32(p.precision)
            wo = int(np.float32(0.5) + np.float32(wo) * P)
            ho = int(np.float32(0.5) + np.float32(ho) * P)
        n = len(inputs)
        nin = sum(c.width * c.height for c in inputs)
        dev = lambda *s, dt=torch.float32: torch.full(s, float("nan") if dt == torch.float32 else -1,
                                                        dtype=dt, device="cuda")
        dbg = {
            "warped_uvz": dev(nin * 4),
            "view_color": dev(n, ho, wo, 3),
            "view_depth": dev(n, ho, wo),
            "view_validity": dev(n, ho, wo),
            "blend_color": dev(ho, wo, 3),
            "blend_quality": dev(ho, wo),
            "inpaint_source": dev(ho, wo, 2, dt=torch.int32),
        }
        sc.synthesize_debug(target, p, out, dbg)
        wo, ho = ow, oh
    else:
        sc.synthesize(target, p, out)
    torch.cuda.synchronize()
    yuv = (to_u16(out[0], (ho, wo)), to_u16(out[1], (ho // 2, wo // 2)), to_u16(out[2], (ho // 2, wo // 2)))
    if debug:
        d = {k: v.cpu().numpy() for k, v in dbg.items()}
        off = 0
        warped = []
        for c in inputs:
            n = c.width * c.height
            warped.append(d["warped_uvz"][off * 4:(off + n) * 4].reshape(c.height, c.width, 4))
            off += n
        d["warped"] = warped
        return yuv, d, sc
    return yuv, sc


def psnr(a, b, peak=1023.0):
    m = np.mean((a.astype(np.float64) - b.astype(np.float64)) ** 2)
    return float("inf") if m == 0 else 10 * np.log10(peak * peak / m)


def parity_report(gpu_yuv, cpu_yuv):
    """PSNR per plane and the fraction of samples differing by more than 2 codes."""
    out = {}
    total = 0
    big = 0
    for name, g, c in zip("YUV", gpu_yuv, cpu_yuv):
        out["psnr_" + name] = psnr(g, c)
        d = np.abs(g.astype(np.int32) - c.astype(np.int32))
        big += int((d > 2).sum())
        total += d.size
        out["maxdiff_" + name] = int(d.max())
    out["frac_gt2"] = big / total
    return out


def assert_parity(gpu_yuv, cpu_yuv, min_psnr=50.0, max_frac=0.005):
    r = parity_report(gpu_yuv, cpu_yuv)
    for k in ("psnr_Y", "psnr_U", "psnr_V"):
        assert r[k] >= min_psnr, r
    assert r["frac_gt2"] <= max_frac, r
    return r
