"""Host-side checks of librvsb.so that need no GPU: the exported C ABI, the
configuration front end (Config.cpp, JsonParser.cpp, PoseTraces.cpp of the
reference) and argument validation of the synthesis entry points."""
import ctypes
import json
import math
import os
import re

import numpy as np
import pytest

import rvsb
from rvsb import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _header_functions():
    text = open(os.path.join(ROOT, "include", "rvsb.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(rvsb_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_function():
    L = rvsb.load()
    declared = _header_functions()
    assert declared, "no declarations found"
    missing = [f for f in declared if not hasattr(L, f)]
    assert not missing, missing
    assert sorted(rvsb.EXPORTED) == declared


def test_struct_sizes_match_header():
    # rvsb_camera: 8 int32 + 16 floats; rvsb_view_planes / yuv420: pointers
    assert ctypes.sizeof(abi.Camera) == 8 * 4 + 16 * 4
    assert ctypes.sizeof(abi.ViewPlanes) == 4 * ctypes.sizeof(ctypes.c_void_p)
    assert ctypes.sizeof(abi.Yuv420) == 3 * ctypes.sizeof(ctypes.c_void_p)
    assert ctypes.sizeof(abi.SynthParams) == 32


def test_status_strings_and_stage_names():
    L = rvsb.load()
    for st in range(10):
        assert L.rvsb_status_string(st)
    assert L.rvsb_status_string(0).decode().lower() in ("ok", "success")
    names = [L.rvsb_stage_name(i).decode() for i in range(len(rvsb.STAGES))]
    assert names == rvsb.STAGES


def test_create_without_device_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    with pytest.raises(rvsb.RvsbError) as e:
        rvsb.Context(0)
    assert e.value.status != 0


@pytest.mark.parametrize("w,h", [(97, 54), (96, 55), (1, 2), (2, 1), (0, 10), (32770, 2), (-4, 8)])
def test_noalloc_rejects_sizes_before_device_work(w, h):
    """Odd sides, sides below 2 and sides above 32768 fail with RVSB_E_ARG
    before any device call (the pointers are never dereferenced), so this
    runs without a GPU."""
    with pytest.raises(rvsb.RvsbError) as e:
        rvsb.inpaint_sources_noalloc(0x1000, w, h, 0x2000)
    assert e.value.status == abi.RVSB_E_ARG
    assert "each side even, 2..32768" in str(e.value)


# ---------------------------------------------------------------------------
# Camera parameters (Parameters.cpp)
# ---------------------------------------------------------------------------

def _persp(**kw):
    d = {"Name": "v", "Projection": "Perspective", "Position": [1, 2, 3], "Rotation": [10, -20, 30],
         "Depthmap": 1, "Background": 0, "Depth_range": [0.5, 100.0], "Resolution": [1920, 1080],
         "Focal": [1500, 1501], "Principle_point": [960, 540], "BitDepthColor": 10, "BitDepthDepth": 16,
         "ColorSpace": "YUV420", "DepthColorSpace": "YUV420"}
    d.update(kw)
    return d


def _erp(**kw):
    d = {"Name": "e", "Projection": "Equirectangular", "Position": [0, 0, 0], "Rotation": [0, 0, 0],
         "Depthmap": 1, "Background": 0, "Depth_range": [0.1, 500.0], "Resolution": [4096, 2048],
         "Hor_range": [-180, 180], "Ver_range": [-90, 90], "BitDepthColor": 10, "BitDepthDepth": 16,
         "ColorSpace": "YUV420", "DepthColorSpace": "YUV420"}
    d.update(kw)
    return d


def test_camera_from_json_perspective():
    c = rvsb.camera_from_json(json.dumps(_persp(HasInvalidDepth=True)))
    assert c.projection == abi.PERSPECTIVE
    assert (c.width, c.height) == (1920, 1080)
    assert list(c.position) == [1, 2, 3]
    assert list(c.rotation) == [10, -20, 30]
    assert list(c.focal) == [1500, 1501]
    assert list(c.principle_point) == [960, 540]
    assert list(c.depth_range) == pytest.approx([0.5, 100.0])
    assert (c.bit_depth_color, c.bit_depth_depth, c.has_invalid_depth) == (10, 16, 1)
    assert c.depth_color_format == abi.YUV420


def test_camera_from_json_erp_full_range():
    c = rvsb.camera_from_json(json.dumps(_erp()))
    assert c.projection == abi.EQUIRECTANGULAR
    assert c.full_hor_range == 1
    c2 = rvsb.camera_from_json(json.dumps(_erp(Hor_range=[-90, 90])))
    assert c2.full_hor_range == 0
    c3 = rvsb.camera_from_json(json.dumps(_erp(DepthColorSpace="YUV400")))
    assert c3.depth_color_format == abi.YUV400


@pytest.mark.parametrize("bad,fragment", [
    (dict(Projection="Fisheye"), "projection"),
    (dict(Depth_range=[10.0, 1.0]), "depth range"),
    (dict(ColorSpace="RGB"), "YUV420"),
    (dict(Depthmap=0), "Depthmap"),
    (dict(Resolution=[1920]), "vector"),
    (dict(BitDepthColor=10.4), "integer"),
])
def test_camera_from_json_rejects(bad, fragment):
    with pytest.raises(rvsb.RvsbError) as e:
        rvsb.camera_from_json(json.dumps(_persp(**bad)))
    assert fragment.lower() in str(e.value).lower()


def test_as_int_rounds_to_nearest():
    """Node::asInt (JsonParser.cpp:303-314) rejects only a positive
    rounding error: 10.5 rounds to 11 and is accepted, 10.4 is not."""
    c = rvsb.camera_from_json(json.dumps(_persp(BitDepthColor=10.5, BitDepthDepth=15.9999999)))
    assert c.bit_depth_color == 11 and c.bit_depth_depth == 16


def test_camera_from_json_missing_key():
    d = _persp()
    del d["Focal"]
    with pytest.raises(rvsb.RvsbError) as e:
        rvsb.camera_from_json(json.dumps(d))
    assert "Focal" in str(e.value)


@pytest.mark.parametrize("extra", [dict(DisplacementMethod="Polynomial"), dict(Crop_region=[0, 0, 960, 540])])
def test_camera_from_json_unsupported(extra):
    """A single camera outside a configuration: a crop region is only
    supported where its padded resolution can be reported (a
    configuration's cameras)."""
    with pytest.raises(rvsb.RvsbError) as e:
        rvsb.camera_from_json(json.dumps(_persp(**extra)))
    assert e.value.status == 7  # RVSB_E_UNSUPPORTED


# ---------------------------------------------------------------------------
# Configuration files (Config.cpp, PoseTraces.cpp)
# ---------------------------------------------------------------------------

def _write_setup(tmp, pose_trace=None, viewport=None, input_extra=None, **over):
    vp = dict(Name="viewport", Resolution=[960, 540], Focal=[750, 750], Principle_point=[480, 270])
    vp.update(viewport or {})
    cams = {"Version": "2.0", "cameras": [_persp(Name="v1", **(input_extra or {})),
                                         _persp(Name="v2", Position=[0, 1, 0]), _persp(**vp)]}
    (tmp / "cams.json").write_text(json.dumps(cams))
    cfg = {"Version": "3.0", "InputCameraParameterFile": "cams.json", "VirtualCameraParameterFile": "cams.json",
           "InputCameraNames": ["v1", "v2"], "VirtualCameraNames": ["viewport"],
           "ViewImageNames": ["t1.yuv", "t2.yuv"], "DepthMapNames": ["d1.yuv", "d2.yuv"],
           "OutputFiles": ["out.yuv"], "NumberOfFrames": 3, "StartFrame": 1, "BlendingFactor": 2.5,
           "Precision": 1.0}
    if pose_trace is not None:
        (tmp / "pose.csv").write_text(pose_trace)
        cfg["VirtualPoseTraceName"] = "pose.csv"
    cfg.update(over)
    cfg = {k: v for k, v in cfg.items() if v is not None}
    (tmp / "rvs.json").write_text(json.dumps(cfg))
    return str(tmp / "rvs.json")


def test_config_load(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    c = rvsb.Config(_write_setup(tmp_path))
    ins = c.inputs()
    assert len(ins) == 2 and list(ins[1].position) == [0, 1, 0]
    v = c.virtual(0)
    assert (v.width, v.height) == (960, 540)
    assert c.frames() == (1, 3, 3)
    p = c.synth_params()
    assert p.blending_factor == 2.5 and p.precision == 1.0 and p.chroma_rounding == 0
    assert c.paths(0) == ("t1.yuv", "d1.yuv")
    assert c.output_path(0) == "out.yuv"


def test_config_precision(tmp_path, monkeypatch):
    """'Precision' reaches the synthesis parameters (Config.cpp:389-399)."""
    monkeypatch.chdir(tmp_path)
    c = rvsb.Config(_write_setup(tmp_path, Precision=2.0))
    assert c.synth_params().precision == 2.0


def test_config_virtual_crop(tmp_path, monkeypatch):
    """Crop_region of the virtual camera: the camera takes the region's size
    and its principal point moves by the region's corner (Parameters.cpp:
    187-190, 245-249); the region and padded size are reported."""
    monkeypatch.chdir(tmp_path)
    c = rvsb.Config(_write_setup(tmp_path, viewport=dict(Crop_region=[100, 50, 640, 360])))
    v = c.virtual(0)
    assert (v.width, v.height) == (640, 360)
    assert list(v.principle_point) == [380.0, 220.0]
    assert c.virtual_crop(0) == ((100, 50, 640, 360), (960, 540))
    full = rvsb.Config(_write_setup(tmp_path))
    assert full.virtual_crop(0) == ((0, 0, 960, 540), (960, 540))


@pytest.mark.parametrize("where,region,status", [
    ("input", [1200, 0, 800, 400], 2),   # outside the resolution
    ("viewport", [400, 0, 640, 360], 2),
    ("viewport", [0, 0, 0, 360], 2),
])
def test_config_crop_rejected(tmp_path, monkeypatch, where, region, status):
    monkeypatch.chdir(tmp_path)
    kw = dict(viewport=dict(Crop_region=region)) if where == "viewport" else dict(input_extra=dict(Crop_region=region))
    with pytest.raises(rvsb.RvsbError) as e:
        rvsb.Config(_write_setup(tmp_path, **kw))
    assert e.value.status == status


def test_config_input_crop(tmp_path, monkeypatch):
    """Crop_region of an input camera: the camera takes the region's size
    and moved principal point, as a virtual camera does, and the region
    and padded size are reported for the loader (colour frames of the
    region's size, depth frames of the padded size)."""
    monkeypatch.chdir(tmp_path)
    res = _persp()["Resolution"]
    pp = _persp()["Principle_point"]
    c = rvsb.Config(_write_setup(tmp_path, input_extra=dict(Crop_region=[64, 32, 800, 400])))
    v1, v2 = c.inputs()
    assert (v1.width, v1.height) == (800, 400)
    assert list(v1.principle_point) == [pp[0] - 64, pp[1] - 32]
    assert c.input_crop(0) == ((64, 32, 800, 400), tuple(res))
    assert c.input_crop(1) == ((0, 0, res[0], res[1]), tuple(res))
    with pytest.raises(rvsb.RvsbError):
        c.input_crop(2)


def test_crop_depth_plane():
    """The region-sized depth map of a cropped input: the padded frame's
    first width * height samples in memory order, not the region's window."""
    padded = np.arange(8 * 6, dtype=np.uint16).reshape(6, 8)
    d = rvsb.crop_depth_plane(padded, 4, 3)
    np.testing.assert_array_equal(d, np.arange(12, dtype=np.uint16).reshape(3, 4))
    with pytest.raises(ValueError):
        rvsb.crop_depth_plane(padded, 8, 7)


def test_config_input_crop_full_resolution(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    res = _persp()["Resolution"]
    c = rvsb.Config(_write_setup(tmp_path, input_extra=dict(Crop_region=[0, 0, res[0], res[1]])))
    assert (c.inputs()[0].width, c.inputs()[0].height) == tuple(res)


def test_config_overrides(tmp_path, monkeypatch):
    """Test_JsonParser_overrides (unit_test.cpp:344-368): keys of the
    override object replace the file's; the others stay."""
    monkeypatch.chdir(tmp_path)
    c = rvsb.Config(_write_setup(tmp_path, InputOverrides={"Depth_range": [1.0, 50.0]},
                                 VirtualOverrides={"Resolution": [480, 270]}))
    assert list(c.inputs()[0].depth_range) == [1.0, 50.0]
    assert list(c.inputs()[0].focal) == [1500, 1501]
    v = c.virtual(0)
    assert (v.width, v.height) == (480, 270)


def test_pose_trace(tmp_path, monkeypatch):
    """Rows of Test_PoseTrace_loadFrom (unit_test.cpp:370-388), applied the
    way Pipeline::computeView does (position += trace, rotation = trace)."""
    monkeypatch.chdir(tmp_path)
    trace = ("X,Y,Z,Yaw,Pitch,Roll\n"
             "0, 0, 0, 7.744e-06, 1.10991e-05, 2.98821e-06\n"
             "-0.000289001, -4.49e-05, -2.50004e-05, -1337, 0.0172351, 0.00275806\n"
             "-0.00062, -8.20999e-05, 1.0, 13.1, 42, 0.00589616\n"
             "-0.047839, 0.0798379, -0.030835, -68.9187, -3.20608, 16.5\n\n")
    c = rvsb.Config(_write_setup(tmp_path, pose_trace=trace))
    base = list(_persp()["Position"])
    f0, f1, f2, f3 = (c.virtual(0, k) for k in range(4))
    assert f0.position[0] == np.float32(base[0]) + np.float32(0.0)
    assert abs(f1.position[1] - (np.float32(base[1]) + np.float32(-4.49e-05))) < 1e-6
    assert f2.position[2] == np.float32(base[2]) + np.float32(1.0)
    assert f1.rotation[0] == -1337.0
    assert f2.rotation[1] == 42.0
    assert f3.rotation[2] == 16.5
    with pytest.raises(rvsb.RvsbError):
        c.virtual(0, 4)


def test_pose_trace_too_short(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    trace = "X,Y,Z,Yaw,Pitch,Roll\n0,0,0,0,0,0\n0,0,0,0,0,0\n"
    with pytest.raises(rvsb.RvsbError) as e:
        rvsb.Config(_write_setup(tmp_path, pose_trace=trace))
    assert "pose trace" in str(e.value)


def test_pose_trace_bad_header(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    with pytest.raises(rvsb.RvsbError):
        rvsb.Config(_write_setup(tmp_path, pose_trace="A,B,C\n0,0,0\n"))


@pytest.mark.parametrize("over,status", [
    (dict(Precision=-1.0), 2),
    (dict(BlendingMethod="Multispectral", BlendingLowFreqFactor=1.0), 2),
    (dict(BlendingMethod="Median"), 2),
    (dict(ViewSynthesisMethod="Squares"), 2),
    (dict(Version="1.0"), 2),
    (dict(DepthMapNames=["d1.yuv"]), 2),
    (dict(InputCameraNames=["v1", "nope"]), 2),
    (dict(InputCameraParameterFile="missing.json"), 3),
])
def test_config_errors(tmp_path, monkeypatch, over, status):
    monkeypatch.chdir(tmp_path)
    with pytest.raises(rvsb.RvsbError) as e:
        rvsb.Config(_write_setup(tmp_path, **over))
    assert e.value.status == status


def test_relative_pose_identity_and_translation():
    a = abi.make_camera(position=(1.0, 2.0, 3.0), rotation=(0, 0, 0))
    b = abi.make_camera(position=(0.0, 0.0, 0.0), rotation=(0, 0, 0))
    R, t = rvsb.relative_pose(a, b)
    assert R == [1, 0, 0, 0, 1, 0, 0, 0, 1]
    assert t == [1.0, 2.0, 3.0]
    c = abi.make_camera(position=(0.0, 0.0, 0.0), rotation=(90, 0, 0))
    R, t = rvsb.relative_pose(a, c)
    # seen from a camera yawed by 90 degrees, +x of the world is -y
    assert np.allclose(np.array(R).reshape(3, 3) @ [1, 0, 0], [0, -1, 0], atol=1e-6)
    assert np.allclose(t, [2.0, -1.0, 3.0], atol=1e-6)


def test_pipeline_header_compiles(tmp_path):
    """include/rvsb_pipeline.hpp (the reference's Pipeline hook points over
    the C ABI) is self-contained: a class deriving from it with the two
    required hooks compiles."""
    import shutil
    import subprocess
    if not shutil.which("g++"):
        pytest.skip("no C++ compiler")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = tmp_path / "p.cpp"
    src.write_text("""
#include "rvsb_pipeline.hpp"
struct App : rvsb::Pipeline {
    rvsb_config* cfg = nullptr;
    const rvsb_config* getConfig() const override { return cfg; }
    rvsb::InputPlanes loadInputView(int, int, const rvsb_camera&) override { return {}; }
    bool wantColor() override { return true; }
    void saveColor(const uint16_t*, int, int, const rvsb_camera&) override {}
};
int main() { App a; (void)a; return 0; }
""")
    cuda_inc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-Wall", "-Wextra", "-I", os.path.join(root, "include"),
                        "-I", cuda_inc, str(src)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
