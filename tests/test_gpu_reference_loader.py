"""The oracle's loader formulas against the reference's own loader on a
B200: read_color / read_depth (rvs/src/image_loading.cpp:74-211) with the
loader kernels of rvs_cuda_lib/src/process_input_frame.cu (resizeUV,
mergeYUV, normalize), compiled unmodified for sm_100a with nvcc's default
contraction into oracle/_ref/libref.so.

Checked bit for bit: the 2x chroma upsample and colour scale, and the depth
decode with its fused multiply-add (z = far*near / fma(d, far-near, near)),
for 10-, 12- and 16-bit depth, YUV420 and YUV400 depth files, HasInvalidDepth
and far >= 1000, and the frame offset with its wrap past the end of file.

Each load runs in a fresh process: the reference's loaders fix their colour
and depth scale at their first call in a process (static const,
image_loading.cpp:134, 193).  test_loader_scale_fixed_by_first_call records
that behaviour with inputs of mixed bit depths; the oracle and the CUDA path
scale every view by its own bit depth instead.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import oracle as O
import ref
from rvsb import abi, scenes

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref.available(), reason="reference harness not built")]

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

_CHILD = r"""
import json, sys
import numpy as np
sys.path.insert(0, {oracle!r}); sys.path.insert(0, {pkg!r})
import ref
from rvsb import abi
jobs = json.load(open(sys.argv[1]))
out = {{}}
for k, job in enumerate(jobs):
    cam = abi.Camera.from_buffer_copy(bytes.fromhex(job["camera"]))
    c, d = ref.load_view(cam, job["color"], job["depth"], job["frame"])
    out[f"c{{k}}"] = c
    out[f"d{{k}}"] = d
np.savez(sys.argv[2], **out)
"""


def _load_in_fresh_process(tmp_path, jobs):
    """[(camera, color_path, depth_path, frame)] -> [(colour, depth)] from
    the reference's loader, all in one new process (first call first)."""
    spec = [{"camera": bytes(c).hex(), "color": cp, "depth": dp, "frame": f} for c, cp, dp, f in jobs]
    jf = tmp_path / "jobs.json"
    jf.write_text(json.dumps(spec))
    out = tmp_path / "out.npz"
    script = _CHILD.format(oracle=os.path.join(ROOT, "oracle"), pkg=os.path.join(ROOT, "rvs-cuda_b200"))
    r = subprocess.run([sys.executable, "-c", script, str(jf), str(out)], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    z = np.load(out)
    return [(z[f"c{k}"], z[f"d{k}"]) for k in range(len(jobs))]


def _write_view(tmp_path, name, planes, frames, depth_format, color_max=1023):
    """Colour (YUV420) and depth (YUV420 with neutral chroma, or YUV400)
    files holding `frames` frames; frame k's luma is shifted by 5k codes."""
    y, u, v, d = planes
    cpath = tmp_path / f"{name}_color.yuv"
    dpath = tmp_path / f"{name}_depth.yuv"
    with open(cpath, "wb") as f:
        for k in range(frames):
            f.write(np.clip(y.astype(np.int32) + 5 * k, 0, color_max).astype("<u2").tobytes())
            f.write(u.astype("<u2").tobytes())
            f.write(v.astype("<u2").tobytes())
    with open(dpath, "wb") as f:
        for k in range(frames):
            f.write(d.astype("<u2").tobytes())
            if depth_format == abi.YUV420:
                c = np.full((d.shape[0] // 2, d.shape[1] // 2), 1 << 15, "<u2")
                f.write(c.tobytes())
                f.write(c.tobytes())
    return str(cpath), str(dpath)


def _frame_luma(y, k):
    return np.clip(y.astype(np.int32) + 5 * k, 0, 1023).astype(np.uint16)


@pytest.mark.parametrize("bits,far,invalid,fmt", [
    (16, 10.0, True, abi.YUV420),
    (16, 10.0, False, abi.YUV400),
    (12, 8.0, True, abi.YUV420),
    (10, 10.0, True, abi.YUV400),
    (16, 1000.0, True, abi.YUV420),
], ids=["d16", "d16_400_valid", "d12", "d10_400", "far1000"])
def test_loader_matches_oracle(tmp_path, bits, far, invalid, fmt):
    wl = scenes.random_pose_small(n_views=1, w=96, h=54, seed=31)
    cam = wl.inputs[0].copy()
    cam.bit_depth_depth = bits
    cam.depth_range[1] = far
    cam.has_invalid_depth = 1 if invalid else 0
    cam.depth_color_format = fmt
    y, u, v, d = wl.planes[0]
    d = (d.astype(np.uint32) >> (16 - bits)).astype(np.uint16)
    d[::7, ::5] = 0  # invalid samples (depth 0 -> NaN when HasInvalidDepth)
    cp, dp = _write_view(tmp_path, "v", (y, u, v, d), 3, fmt)
    # frames 0 and 2, and 5: past the end of the file, which reads frame 0
    got = _load_in_fresh_process(tmp_path, [(cam, cp, dp, 0), (cam, cp, dp, 2), (cam, cp, dp, 5)])
    for (c, dd), k in zip(got, (0, 2, 0)):
        np.testing.assert_array_equal(c, O.decode_color(_frame_luma(y, k), u, v, cam.bit_depth_color))
        np.testing.assert_array_equal(dd, O.decode_depth(d, cam))


def test_loader_scale_fixed_by_first_call(tmp_path):
    """Two views of different colour and depth bit depths loaded in one
    process: the second is scaled with the first one's levels
    (1/1023 and 1/65535), not its own (1/4095 and 1/4095)."""
    wl = scenes.random_pose_small(n_views=2, w=64, h=36, seed=32)
    a, b = wl.inputs[0].copy(), wl.inputs[1].copy()
    b.bit_depth_color = 12
    b.bit_depth_depth = 12
    ya, ua, va, da = wl.planes[0]
    yb, ub, vb, db = wl.planes[1]
    yb, ub, vb = (x.astype(np.uint16) * 4 for x in (yb, ub, vb))
    db = (db >> 4).astype(np.uint16)
    pa = _write_view(tmp_path, "a", (ya, ua, va, da), 1, abi.YUV420)
    pb = _write_view(tmp_path, "b", (yb, ub, vb, db), 1, abi.YUV420, color_max=4095)
    (ca, _), (cb, dbr) = _load_in_fresh_process(tmp_path, [(a, *pa, 0), (b, *pb, 0)])
    np.testing.assert_array_equal(ca, O.decode_color(ya, ua, va, 10))
    # the reference: b's samples scaled by a's 10-bit colour level ...
    b_as_10 = O.decode_color(yb, ub, vb, 10)
    np.testing.assert_array_equal(cb, b_as_10)
    # ... which the oracle (own bit depth per view) does not do
    assert not np.array_equal(cb, O.decode_color(yb, ub, vb, 12))
    # depth: b's 12-bit samples scaled by 1/65535 (a's 16-bit level)
    b16 = b.copy()
    b16.bit_depth_depth = 16
    np.testing.assert_array_equal(dbr, O.decode_depth(db, b16))
