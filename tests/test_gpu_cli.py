"""The RVS drop-in CLI (rvs-cuda_b200/lib/rvsb) end to end: reference-format
configuration, camera file, pose trace and raw YUV files in, the five output
files out, every output frame checked against the oracle.  Three input
frames and five output frames exercise the ping-pong frame index
(Pipeline.cpp:157-167) and the pose trace (Pipeline.cpp:173-181)."""
import copy
import json
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from rvsb import abi, scenes
from helpers import assert_parity

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "rvs-cuda_b200", "lib", "rvsb")


def _cam_json(name, c):
    d = {"Name": name, "Projection": "Equirectangular" if c.projection else "Perspective",
         "Position": [float(x) for x in c.position], "Rotation": [float(x) for x in c.rotation],
         "Depthmap": 1, "Background": 0, "Depth_range": [float(x) for x in c.depth_range],
         "Resolution": [c.width, c.height], "BitDepthColor": c.bit_depth_color, "BitDepthDepth": c.bit_depth_depth,
         "ColorSpace": "YUV420", "DepthColorSpace": "YUV420", "HasInvalidDepth": bool(c.has_invalid_depth)}
    if c.projection:
        d["Hor_range"] = [float(x) for x in c.hor_range]
        d["Ver_range"] = [float(x) for x in c.ver_range]
    else:
        d["Focal"] = [float(x) for x in c.focal]
        d["Principle_point"] = [float(x) for x in c.principle_point]
    return d


def _frame_planes(planes, k):
    """Input frame k: luma shifted by 7 codes per frame so frames differ."""
    y, u, v, d = planes
    y2 = np.clip(y.astype(np.int32) + 7 * k, 0, 1023).astype(np.uint16)
    return y2, u, v, d


def extended_index(f, n):
    g, r = divmod(f, n)
    return n - r - 1 if g % 2 else r


def test_cli_end_to_end(tmp_path):
    wl = scenes.random_pose_small(n_views=2, w=96, h=54, seed=91)
    n_frames, n_out = 3, 5
    names = [f"v{i}" for i in range(len(wl.inputs))]
    target = wl.targets[0]
    cams = {"Version": "2.0", "cameras": [_cam_json(n, c) for n, c in zip(names, wl.inputs)] +
            [_cam_json("viewport", target)]}
    (tmp_path / "cams.json").write_text(json.dumps(cams))
    for i, planes in enumerate(wl.planes):
        with open(tmp_path / f"t{i}.yuv", "wb") as ft, open(tmp_path / f"d{i}.yuv", "wb") as fd:
            for k in range(n_frames):
                y, u, v, d = _frame_planes(planes, k)
                ft.write(y.tobytes() + u.tobytes() + v.tobytes())
                chroma = np.full((d.shape[0] // 2) * (d.shape[1] // 2), 32768, np.uint16)
                fd.write(d.tobytes() + chroma.tobytes() + chroma.tobytes())
    rng = np.random.default_rng(5)
    trace = []
    for f in range(n_out):
        dp = rng.uniform(-0.01, 0.01, 3)
        rot = [target.rotation[0] + rng.uniform(-1, 1), target.rotation[1], target.rotation[2]]
        trace.append((dp, rot))
    (tmp_path / "pose.csv").write_text("X,Y,Z,Yaw,Pitch,Roll\n" + "".join(
        ",".join(repr(float(x)) for x in list(dp) + list(rot)) + "\n" for dp, rot in trace))
    cfg = {"Version": "3.0", "InputCameraParameterFile": "cams.json", "VirtualCameraParameterFile": "cams.json",
           "InputCameraNames": names, "VirtualCameraNames": ["viewport"],
           "ViewImageNames": [f"t{i}.yuv" for i in range(len(names))],
           "DepthMapNames": [f"d{i}.yuv" for i in range(len(names))],
           "OutputFiles": ["out.yuv"], "MaskedOutputFiles": ["masked.yuv"], "OutputMasks": ["mask.yuv"],
           "DepthOutputFiles": ["depth.yuv"], "MaskedDepthOutputFiles": ["mdepth.yuv"],
           "NumberOfFrames": n_frames, "NumberOfOutputFrames": n_out, "StartFrame": 0,
           "VirtualPoseTraceName": "pose.csv", "BlendingFactor": 5.0, "ValidityThreshold": 6000.0}
    (tmp_path / "rvs.json").write_text(json.dumps(cfg))
    r = subprocess.run([CLI, "rvs.json", "--cuda"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    wo, ho = target.width, target.height
    ny, nc = wo * ho, (wo // 2) * (ho // 2)
    out = np.fromfile(tmp_path / "out.yuv", np.uint16).reshape(n_out, ny + 2 * nc)
    masked = np.fromfile(tmp_path / "masked.yuv", np.uint16).reshape(n_out, ny + 2 * nc)
    mask = np.fromfile(tmp_path / "mask.yuv", np.uint8).reshape(n_out, ny + 2 * nc)
    depth = np.fromfile(tmp_path / "depth.yuv", np.uint16).reshape(n_out, ny + 2 * nc)
    mdepth = np.fromfile(tmp_path / "mdepth.yuv", np.uint16).reshape(n_out, ny + 2 * nc)
    assert (mask[:, ny:] == 128).all() and (depth[:, ny:] == 32768).all()
    for f in range(n_out):
        k = extended_index(f, n_frames)
        planes = [_frame_planes(p, k) for p in wl.planes]
        virt = copy.deepcopy(target)
        dp, rot = trace[f]
        for a in range(3):
            virt.position[a] = np.float32(np.float32(target.position[a]) + np.float32(dp[a]))
            virt.rotation[a] = np.float32(rot[a])
        ref = O.synthesize_aux(wl.inputs, planes, virt, 5.0, 6000.0)
        got = O.split_yuv420(out[f], wo, ho)
        assert_parity(got, ref["yuv"])
        assert_parity(O.split_yuv420(masked[f], wo, ho), ref["masked_yuv"])
        assert (mask[f, :ny].reshape(ho, wo) != ref["mask"]).mean() <= 1e-3
        for g, rr in ((depth[f, :ny], ref["depth"]), (mdepth[f, :ny], ref["masked_depth"])):
            diff = np.abs(g.reshape(ho, wo).astype(np.int64) - rr.astype(np.int64))
            assert (diff > 1).mean() <= 5e-3


def test_cli_crop_region(tmp_path, monkeypatch):
    """A virtual camera with Crop_region: the colour output has the region's
    size and matches the oracle's synthesis of the cropped camera; the mask
    and depth outputs have the padded resolution with an all-zero luma
    plane, as the reference's writers produce them (their
    `padded(region) = image` copies nothing, image_writing.cpp:262-267,
    285-290): checked against those writers where the reference harness is
    built."""
    wl = scenes.random_pose_small(n_views=2, w=96, h=54, seed=93)
    names = [f"v{i}" for i in range(len(wl.inputs))]
    target = wl.targets[0]
    cx, cy, pw, ph = 16, 8, target.width + 32, target.height + 18
    vp = _cam_json("viewport", target)
    vp["Resolution"] = [pw, ph]
    vp["Crop_region"] = [cx, cy, target.width, target.height]
    vp["Principle_point"] = [float(target.principle_point[0]) + cx, float(target.principle_point[1]) + cy]
    cams = {"Version": "2.0", "cameras": [_cam_json(n, c) for n, c in zip(names, wl.inputs)] + [vp]}
    (tmp_path / "cams.json").write_text(json.dumps(cams))
    for i, planes in enumerate(wl.planes):
        y, u, v, d = planes
        (tmp_path / f"t{i}.yuv").write_bytes(y.tobytes() + u.tobytes() + v.tobytes())
        chroma = np.full((d.shape[0] // 2) * (d.shape[1] // 2), 32768, np.uint16)
        (tmp_path / f"d{i}.yuv").write_bytes(d.tobytes() + chroma.tobytes() + chroma.tobytes())
    cfg = {"Version": "3.0", "InputCameraParameterFile": "cams.json", "VirtualCameraParameterFile": "cams.json",
           "InputCameraNames": names, "VirtualCameraNames": ["viewport"],
           "ViewImageNames": [f"t{i}.yuv" for i in range(len(names))],
           "DepthMapNames": [f"d{i}.yuv" for i in range(len(names))],
           "OutputFiles": ["out.yuv"], "OutputMasks": ["mask.yuv"], "DepthOutputFiles": ["depth.yuv"],
           "NumberOfFrames": 1, "BlendingFactor": 5.0, "ValidityThreshold": 6000.0}
    (tmp_path / "rvs.json").write_text(json.dumps(cfg))
    import rvsb
    monkeypatch.chdir(tmp_path)  # camera files are resolved against the working directory
    virt = rvsb.Config("rvs.json").virtual(0)
    assert (virt.width, virt.height) == (target.width, target.height)
    r = subprocess.run([CLI, "rvs.json"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    wo, ho = target.width, target.height
    ref = O.synthesize_aux(wl.inputs, wl.planes, virt, 5.0, 6000.0)
    out = np.fromfile(tmp_path / "out.yuv", np.uint16)
    assert out.size == wo * ho * 3 // 2
    assert_parity(O.split_yuv420(out, wo, ho), ref["yuv"])
    npy = pw * ph
    mask = np.fromfile(tmp_path / "mask.yuv", np.uint8)
    depth = np.fromfile(tmp_path / "depth.yuv", np.uint16)
    assert mask.size == npy * 3 // 2 and depth.size == npy * 3 // 2
    assert (mask[npy:] == 128).all() and (depth[npy:] == 32768).all()
    my, dy = mask[:npy].reshape(ph, pw), depth[:npy].reshape(ph, pw)
    assert not my.any() and not dy.any()
    import ref as R
    if R.available():
        crop, padded = (cx, cy, wo, ho), (pw, ph)
        rmask = R.write_aux("mask", None, (ref["mask"] != 0).astype(np.uint8), virt, crop, padded)
        rdepth = R.write_aux("depth", np.full((ho, wo), 2.0, np.float32), None, virt, crop, padded)
        np.testing.assert_array_equal(my, rmask)
        np.testing.assert_array_equal(dy, rdepth)


def _small_config(tmp_path, wl, n_frames=1):
    names = [f"v{i}" for i in range(len(wl.inputs))]
    cams = {"Version": "2.0", "cameras": [_cam_json(n, c) for n, c in zip(names, wl.inputs)] +
            [_cam_json("viewport", wl.targets[0])]}
    (tmp_path / "cams.json").write_text(json.dumps(cams))
    for i, planes in enumerate(wl.planes):
        y, u, v, d = planes
        (tmp_path / f"t{i}.yuv").write_bytes((y.tobytes() + u.tobytes() + v.tobytes()) * n_frames)
        chroma = np.full((d.shape[0] // 2) * (d.shape[1] // 2), 32768, np.uint16)
        (tmp_path / f"d{i}.yuv").write_bytes((d.tobytes() + chroma.tobytes() + chroma.tobytes()) * n_frames)
    cfg = {"Version": "3.0", "InputCameraParameterFile": "cams.json", "VirtualCameraParameterFile": "cams.json",
           "InputCameraNames": names, "VirtualCameraNames": ["viewport"],
           "ViewImageNames": [f"t{i}.yuv" for i in range(len(names))],
           "DepthMapNames": [f"d{i}.yuv" for i in range(len(names))],
           "OutputFiles": ["out.yuv"], "NumberOfFrames": n_frames, "BlendingFactor": 5.0}
    (tmp_path / "rvs.json").write_text(json.dumps(cfg))


@pytest.mark.parametrize("fault", ["missing_color", "missing_depth", "truncated_color", "truncated_depth"])
def test_cli_input_file_faults(tmp_path, fault):
    """Loader faults as the reference reports them: a missing file fails with
    'Failed to read raw YUV color|depth file "<path>"' (image_loading.cpp:84-90,
    155-161), a file shorter than one frame with 'Failed to read the expected
    amount of data' (image_loading.cpp:66-71); the CLI prints the message and
    exits with status 1 (view_synthesis.cpp:171-175), writing no frame."""
    wl = scenes.random_pose_small(n_views=2, w=64, h=36, seed=95)
    _small_config(tmp_path, wl)
    kind, what = fault.split("_")[1], fault.split("_")[0]
    path = tmp_path / (f"t1.yuv" if kind == "color" else f"d1.yuv")
    if what == "missing":
        path.unlink()
    else:
        path.write_bytes(path.read_bytes()[:1000])
    r = subprocess.run([CLI, "rvs.json"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 1
    if what == "missing":
        assert f'Failed to read raw YUV {kind} file "{path.name}"' in r.stderr, r.stderr
    else:
        assert "Failed to read the expected amount of data" in r.stderr, r.stderr


def test_cli_frames_past_end_wrap(tmp_path):
    """More output frames than the input files hold: each frame index past
    the end of a file reads frame 0 (image_loading.cpp:95-98), so all three
    output frames equal the one-frame synthesis."""
    wl = scenes.random_pose_small(n_views=2, w=64, h=36, seed=96)
    _small_config(tmp_path, wl)
    cfg = json.loads((tmp_path / "rvs.json").read_text())
    cfg["NumberOfFrames"] = 3
    cfg["NumberOfOutputFrames"] = 3
    (tmp_path / "rvs.json").write_text(json.dumps(cfg))
    r = subprocess.run([CLI, "rvs.json"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    t = wl.targets[0]
    n = t.width * t.height * 3 // 2
    out = np.fromfile(tmp_path / "out.yuv", np.uint16).reshape(3, n)
    assert_parity(O.split_yuv420(out[0], t.width, t.height), O.synthesize(wl.inputs, wl.planes, t, 5.0))
    np.testing.assert_array_equal(out[1], out[0])
    np.testing.assert_array_equal(out[2], out[0])


def test_cli_input_crop_region(tmp_path):
    """An input camera with Crop_region, read as the reference reads it:
    colour frames of the region's size (image_loading.cpp:76), depth frames
    of the padded size (image_loading.cpp:149) whose first region-area
    samples, in memory order, are the view's depth (SynthesizedView.cpp:
    89-94).  The padded depth frames hold the true depth there and other
    values in the region's window, so reading the window would fail; two
    frames check the padded frame offset.  The output matches the oracle's
    synthesis of the uncropped inputs, and, where the reference harness is
    built, the reference's own loader gives the same depth."""
    wl = scenes.random_pose_small(n_views=2, w=96, h=54, seed=95)
    names = [f"v{i}" for i in range(len(wl.inputs))]
    target = wl.targets[0]
    c0 = wl.inputs[0]
    w, h = c0.width, c0.height
    cx, cy, pw, ph = 6, 4, w + 10, h + 8
    v0 = _cam_json(names[0], c0)
    v0["Resolution"] = [pw, ph]
    v0["Crop_region"] = [cx, cy, w, h]
    v0["Principle_point"] = [float(c0.principle_point[0]) + cx, float(c0.principle_point[1]) + cy]
    cams = {"Version": "2.0", "cameras": [v0] + [_cam_json(n, c) for n, c in zip(names[1:], wl.inputs[1:])] +
            [_cam_json("viewport", target)]}
    (tmp_path / "cams.json").write_text(json.dumps(cams))
    n_frames = 2
    rng = np.random.default_rng(17)

    def depth_k(d, k):
        return np.clip(d.astype(np.int32) + 300 * k, 0, 65535).astype(np.uint16)

    padded_frames = []
    for i, planes in enumerate(wl.planes):
        y, u, v, d = planes
        with open(tmp_path / f"t{i}.yuv", "wb") as ft, open(tmp_path / f"d{i}.yuv", "wb") as fd:
            for k in range(n_frames):
                yk, uk, vk, _ = _frame_planes(planes, k)
                ft.write(yk.tobytes() + uk.tobytes() + vk.tobytes())
                dk = depth_k(d, k)
                if i == 0:
                    pad = rng.integers(0, 65536, (ph, pw)).astype(np.uint16)
                    pad.reshape(-1)[:w * h] = dk.reshape(-1)
                    padded_frames.append(pad)
                    dk = pad
                chroma = np.full((dk.shape[0] // 2) * (dk.shape[1] // 2), 32768, np.uint16)
                fd.write(dk.tobytes() + chroma.tobytes() + chroma.tobytes())
    window = padded_frames[0][cy:cy + h, cx:cx + w]
    assert (window != wl.planes[0][3]).mean() > 0.5  # the window is not the depth
    cfg = {"Version": "3.0", "InputCameraParameterFile": "cams.json", "VirtualCameraParameterFile": "cams.json",
           "InputCameraNames": names, "VirtualCameraNames": ["viewport"],
           "ViewImageNames": [f"t{i}.yuv" for i in range(len(names))],
           "DepthMapNames": [f"d{i}.yuv" for i in range(len(names))],
           "OutputFiles": ["out.yuv"], "NumberOfFrames": n_frames, "BlendingFactor": 5.0}
    (tmp_path / "rvs.json").write_text(json.dumps(cfg))
    r = subprocess.run([CLI, "rvs.json"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    wo, ho = target.width, target.height
    out = np.fromfile(tmp_path / "out.yuv", np.uint16).reshape(n_frames, -1)
    import rvsb
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        conf = rvsb.Config("rvs.json")
        assert conf.input_crop(0) == ((cx, cy, w, h), (pw, ph))
        cin = conf.inputs()[0]
    finally:
        os.chdir(cwd)
    assert list(cin.principle_point) == list(c0.principle_point)
    for k in range(n_frames):
        planes = []
        for i, p in enumerate(wl.planes):
            yk, uk, vk, _ = _frame_planes(p, k)
            dk = rvsb.crop_depth_plane(padded_frames[k], w, h) if i == 0 else depth_k(p[3], k)
            planes.append((yk, uk, vk, dk))
        np.testing.assert_array_equal(planes[0][3], depth_k(wl.planes[0][3], k))
        ref = O.synthesize(wl.inputs, planes, target, 5.0)
        assert_parity(O.split_yuv420(out[k], wo, ho), ref)
    import ref as R
    if R.available():
        import sys
        script = (f"import sys, numpy as np; sys.path.insert(0, {os.path.join(ROOT, 'oracle')!r}); "
                  f"sys.path.insert(0, {os.path.join(ROOT, 'rvs-cuda_b200')!r}); import ref; from rvsb import abi; "
                  f"cam = abi.Camera.from_buffer_copy(bytes.fromhex(sys.argv[1])); "
                  f"out = [ref.load_view(cam, 't0.yuv', 'd0.yuv', k, ({cx}, {cy}, {w}, {h}), ({pw}, {ph}))[1] "
                  f"for k in range({n_frames})]; np.save(sys.argv[2], np.stack(out))")
        r = subprocess.run([sys.executable, "-c", script, bytes(c0).hex(), str(tmp_path / "rd.npy")], cwd=tmp_path,
                           capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stdout + r.stderr
        rd = np.load(tmp_path / "rd.npy")
        for k in range(n_frames):
            want = O.decode_depth(depth_k(wl.planes[0][3], k), c0)
            np.testing.assert_array_equal(rd[k], want)
