"""The CPU oracle against the golden fixtures (tests/golden/make_golden.py)
and the reference's own unit-test known answers (rvs/src/unit_test.cpp,
rederived analytically as the reference's tests do)."""
import math
import os

import numpy as np
import pytest

import oracle as O
import rvsb
from rvsb import abi

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    return np.load(os.path.join(GOLDEN, name))


# ---------------------------------------------------------------------------
# OpenCV behaviour at the boundary (pinned against the cv2 wheel)
# ---------------------------------------------------------------------------

def _codes_to_color(codes, bits):
    """A float image whose quantised codes (trunc(v * max)) are `codes`."""
    m = float((1 << bits) - 1)
    return ((codes.astype(np.float64) + 0.5) / m).astype(np.float32)


@pytest.mark.parametrize("bits", [10, 16])
@pytest.mark.parametrize("mode,suffix", [(0, ""), (1, "_noipp")], ids=["ipp", "noipp"])
def test_writer_chroma_matches_cv2_resize(bits, mode, suffix):
    """write_color_YUV's cv::resize(0.5, 0.5, INTER_LINEAR) on the quantised
    chroma: mode 0 matches OpenCV with IPP, mode 1 OpenCV without."""
    z = _load("cv2_resize_half.npz")
    cases = [(z[f"in{k}"], z[f"out{k}{suffix}"]) for k in range(int(z["n"]))] if bits == 10 else \
        [(z["full_range_in"], z[f"full_range_out{suffix}"])]
    O.set_chroma_round(mode)
    try:
        for codes, expected in cases:
            h, w = codes.shape
            color = np.zeros((h, w, 3), np.float32)
            color[..., 0] = _codes_to_color(codes, bits)
            color[..., 1] = _codes_to_color(codes, bits)
            flipped = codes[::-1, ::-1].copy()
            color[..., 2] = _codes_to_color(flipped, bits)
            Y, U, V = O.write_yuv420(color, bits)
            np.testing.assert_array_equal(Y, codes)
            np.testing.assert_array_equal(U, expected)
            s = flipped.astype(np.int64)
            s = s[0::2, 0::2] + s[1::2, 0::2] + s[0::2, 1::2] + s[1::2, 1::2]
            q, r = s >> 2, s & 3
            ref = (s + 2) >> 2 if mode else q + ((r > 2) | ((r == 2) & (q & 1 == 1)))
            np.testing.assert_array_equal(V, ref)
    finally:
        O.set_chroma_round(0)


def test_ipp_and_plain_opencv_differ_only_on_ties():
    z = _load("cv2_resize_half.npz")
    for k in range(int(z["n"])):
        a = z[f"in{k}"].astype(np.int64)
        s = a[0::2, 0::2] + a[1::2, 0::2] + a[0::2, 1::2] + a[1::2, 1::2]
        diff = z[f"out{k}"] != z[f"out{k}_noipp"]
        assert np.all(s[diff] % 4 == 2)


def test_edge_norm_matches_cv2():
    """cv::norm(Vec2f, Vec2f) of valid_tri.  OpenCV 4.9 (the version the
    reference was tested on) forms the difference in float and sums its
    squares in double; the cv2 wheel's newer dispatched kernel subtracts in
    double and fuses the last multiply-add.  The two agree exactly whenever
    the float difference is exact, which is the case for the nearby vertex
    positions of a triangle edge; the oracle follows 4.9."""
    z = _load("cv2_norm_vec2f.npz")
    a, b, ref = z["a"], z["b"], z["norm"]
    got = np.array([O.edge_norm(x, y) for x, y in zip(a, b)])
    exact = np.all((a - b).astype(np.float64) == a.astype(np.float64) - b.astype(np.float64), axis=1)
    assert exact.mean() > 0.5
    np.testing.assert_array_equal(got[exact], ref[exact])
    d = (a - b).astype(np.float64)
    np.testing.assert_array_equal(got, np.sqrt(d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]))


def _camera(a):
    c = abi.Camera()
    import ctypes
    ctypes.memmove(ctypes.addressof(c), a.tobytes(), ctypes.sizeof(c))
    return c


@pytest.mark.parametrize("k", [0, 1, 2])
def test_oracle_regression(k):
    z = _load(f"synth_small_{k}.npz")
    n = int(z["n"])
    cams = [_camera(z[f"cam{i}"]) for i in range(n)]
    planes = [(z[f"y{i}"], z[f"u{i}"], z[f"v{i}"], z[f"d{i}"]) for i in range(n)]
    (Y, U, V), q, _ = O.synthesize(cams, planes, _camera(z["target"]), float(z["exponent"]),
                                   want_intermediate=True)
    np.testing.assert_array_equal(Y, z["Y"])
    np.testing.assert_array_equal(U, z["U"])
    np.testing.assert_array_equal(V, z["V"])
    np.testing.assert_array_equal(q > 0, z["quality"] > 0)


# ---------------------------------------------------------------------------
# Camera models: unit_test.cpp:90-308
# ---------------------------------------------------------------------------

ERP_JSON = """{"Name": "v0", "Projection": "Equirectangular", "Position": [0, 0, 0],
 "Rotation": [0, 0, 0], "Depthmap": 1, "Background": 0, "Depth_range": [0, 1],
 "Resolution": [5, 5], "BitDepthColor": 13, "BitDepthDepth": 15, "ColorSpace": "YUV420",
 "DepthColorSpace": "YUV420", "Hor_range": [-180, 180], "Ver_range": [-90, 90]}"""

PERSP_JSON = """{"Name": "v0", "Projection": "Perspective", "Position": [5, 3, 9],
 "Rotation": [10, 5, -3], "Depthmap": 1, "Background": 0, "Depth_range": [0, 1],
 "Resolution": [4, 3], "Focal": [3, 3], "Principle_point": [2, 1], "BitDepthColor": 10,
 "BitDepthDepth": 10, "ColorSpace": "YUV420", "DepthColorSpace": "YUV420"}"""


def _erp_reference():
    pos = np.zeros((5, 5, 2), np.float32)
    for j in range(5):
        pos[:, j, 0] = j + 0.5
    pos[:, :, 1] = np.array([0.001, 1.5, 2.5, 3.5, 4.999], np.float32)[:, None]
    depth = np.ones((5, 5), np.float32)
    depth[2, 2] = 2.0
    world = np.zeros((5, 5, 3), np.float32)
    for i in range(5):
        for j in range(5):
            phi = math.pi - 2 * math.pi * (pos[i, j, 0] / 5.0)
            theta = math.pi / 2 - math.pi * (pos[i, j, 1] / 5.0)
            world[i, j] = [depth[i, j] * math.cos(theta) * math.cos(phi),
                           depth[i, j] * math.cos(theta) * math.sin(phi), depth[i, j] * math.sin(theta)]
    return pos, depth, world


def test_erp_image_pos():
    cam = rvsb.camera_from_json(ERP_JSON)
    pos, _, _ = _erp_reference()
    assert np.abs(O.image_pos(cam) - pos).max() < 1e-6


def test_erp_unproject():
    cam = rvsb.camera_from_json(ERP_JSON)
    pos, depth, world = _erp_reference()
    assert np.abs(O.unproject(cam, pos, depth) - world).max() < 1e-6


def test_erp_project():
    cam = rvsb.camera_from_json(ERP_JSON)
    pos, depth, world = _erp_reference()
    uv, d, wrap = O.project(cam, world)
    assert np.abs(uv - pos).max() < 1e-4
    assert np.abs(d - depth).max() < 1e-6
    assert wrap == 1


def _persp_reference():
    pos = np.zeros((3, 4, 2), np.float32)
    for i in range(3):
        for j in range(4):
            pos[i, j] = [j + 0.5, i + 0.5]
    depth = np.ones((3, 4), np.float32)
    depth[2, 2] = 2.0
    world = np.zeros((3, 4, 3), np.float32)
    for i in range(3):
        for j in range(4):
            sensor = np.array([3.0, 2.0 - pos[i, j, 0], 1.0 - pos[i, j, 1]])
            world[i, j] = (sensor * (depth[i, j] / 3.0)).astype(np.float32)
    return pos, depth, world


def test_perspective_image_pos_unproject_project():
    cam = rvsb.camera_from_json(PERSP_JSON)
    pos, depth, world = _persp_reference()
    assert np.abs(O.image_pos(cam) - pos).max() < 1e-6
    assert np.abs(O.unproject(cam, pos, depth) - world).max() < 1e-6
    uv, d, wrap = O.project(cam, world)
    assert np.abs(uv - pos).max() < 1e-6
    assert np.abs(d - depth).max() < 1e-6
    assert wrap == 0


def test_rotation_matrix_is_rz_ry_rx():
    rot = (23.0, -11.0, 7.5)
    R = O.rotation_matrix(rot)
    a, b, c = (math.radians(x) for x in rot)
    rz = np.array([[math.cos(a), -math.sin(a), 0], [math.sin(a), math.cos(a), 0], [0, 0, 1]])
    ry = np.array([[math.cos(b), 0, math.sin(b)], [0, 1, 0], [-math.sin(b), 0, math.cos(b)]])
    rx = np.array([[1, 0, 0], [0, math.cos(c), -math.sin(c)], [0, math.sin(c), math.cos(c)]])
    np.testing.assert_allclose(R, rz @ ry @ rx, atol=1e-6)


def test_library_relative_pose_matches_oracle():
    rng = np.random.default_rng(7)
    for _ in range(200):
        a = abi.make_camera(position=rng.normal(size=3), rotation=rng.uniform(-180, 180, 3))
        b = abi.make_camera(position=rng.normal(size=3), rotation=rng.uniform(-180, 180, 3))
        R1, t1 = rvsb.relative_pose(a, b)
        R2, t2 = O.relative_pose(a, b)
        np.testing.assert_array_equal(np.array(R1, np.float32), R2.ravel())
        np.testing.assert_array_equal(np.array(t1, np.float32), t2)


def test_depth_decode_formula():
    cam = abi.make_camera(depth_range=(0.5, 10.0), bit_depth_depth=16)
    raw = np.array([[0, 1, 32768, 65535]], np.uint16)
    z = O.decode_depth(raw, cam)
    d = raw.astype(np.float64) / 65535.0
    np.testing.assert_allclose(z, 10 * 0.5 / (0.5 + d * 9.5), rtol=1e-6)
    inf_cam = abi.make_camera(depth_range=(0.5, 1000.0), bit_depth_depth=16)
    zi = O.decode_depth(raw, inf_cam)
    assert np.isinf(zi[0, 0]) and abs(zi[0, 3] - 0.5) < 1e-6
