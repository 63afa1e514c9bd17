"""TEST INFRASTRUCTURE ONLY: ctypes loader for oracle/_ref/libref.so, the
reference's own CPU synthesis code (and its loader kernels) compiled
unmodified against an OpenCV stand-in by oracle/ref/Makefile.

The tests use it to check the oracle (rvs_oracle.cpp) stage by stage against
the reference itself.  The library is built where the reference tree is
present (RVS_REFERENCE, default /root/reference) and travels with the tree as
a built file; nothing here reads the reference's sources at run time.
"""
import ctypes
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "rvs-cuda_b200"))
from rvsb import abi  # noqa: E402

LIB_PATH = os.path.join(HERE, "_ref", "libref.so")
REFERENCE = os.environ.get("RVS_REFERENCE", "/root/reference")

_lib = None

_F = ctypes.POINTER(ctypes.c_float)
_I32 = ctypes.POINTER(ctypes.c_int32)
_U8 = ctypes.POINTER(ctypes.c_uint8)


def reference_tree_present():
    return os.path.isfile(os.path.join(REFERENCE, "rvs", "src", "transform.cpp"))


def build():
    """Builds oracle/_ref/libref.so from the reference tree (a no-op when it
    is up to date).  Returns False when neither the tree nor a built library
    exists."""
    if reference_tree_present():
        subprocess.check_call(["make", "-s", "-j8", "-C", os.path.join(HERE, "ref"), "REF=" + REFERENCE])
    return os.path.exists(LIB_PATH)


def available():
    return os.path.exists(LIB_PATH) or reference_tree_present()


def lib():
    global _lib
    if _lib is None:
        if not build():
            raise RuntimeError("oracle/_ref/libref.so is not built and the reference tree is absent")
        L = ctypes.CDLL(LIB_PATH)
        c_p = ctypes.c_void_p
        L.ref_last_error.restype = ctypes.c_char_p
        L.ref_set_precision.argtypes = [ctypes.c_float]
        L.ref_set_resize_ties_up.argtypes = [ctypes.c_int]
        L.ref_camera_new.argtypes = [ctypes.c_char_p]
        L.ref_camera_new.restype = c_p
        L.ref_camera_free.argtypes = [c_p]
        L.ref_relative_pose.argtypes = [c_p, c_p, _F, _F]
        L.ref_warp.argtypes = [c_p, c_p, _F, _F, _F, ctypes.POINTER(ctypes.c_int)]
        L.ref_raster.argtypes = [_F, _F, _F, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                 _F, _F, _F, _F]
        PF = ctypes.POINTER(_F)
        L.ref_blend.argtypes = [ctypes.c_int, PF, PF, PF, PF, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                ctypes.c_int, ctypes.c_float, ctypes.c_float, _F, _F, _F, _F]
        L.ref_inpaint.argtypes = [_F, _F, ctypes.c_int, ctypes.c_int, _F]
        L.ref_inpaint_sources.argtypes = [_U8, ctypes.c_int, ctypes.c_int, _I32]
        L.ref_write_color.argtypes = [_F, ctypes.c_int, ctypes.c_int, c_p, ctypes.c_char_p]
        L.ref_synthesize.argtypes = [ctypes.c_int, ctypes.POINTER(c_p), PF, PF, c_p, ctypes.c_float, ctypes.c_int,
                                     ctypes.c_float, ctypes.c_float, _F, _F]
        L.ref_load_view.argtypes = [c_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, _F, _F]
        L.ref_write_aux.argtypes = [ctypes.c_int, _F, _U8, ctypes.c_int, ctypes.c_int, c_p, ctypes.c_char_p]
        _lib = L
    return _lib


def _check(rc):
    if rc != 0:
        raise RuntimeError("reference: " + lib().ref_last_error().decode())


def _p(a, t=_F):
    return a.ctypes.data_as(t)


def camera_dict(c, name="cam", crop=None, padded=None):
    """The camera-parameter JSON object of an rvsb camera (the keys of
    Parameters.cpp).  crop=(x, y, w, h) with padded=(W, H): the camera is
    the region of a W x H camera (Crop_region; c holds the region's size
    and its principal point relative to the region)."""
    d = {"Name": name, "Projection": "Equirectangular" if c.projection == abi.EQUIRECTANGULAR else "Perspective",
         "Position": [float(x) for x in c.position], "Rotation": [float(x) for x in c.rotation],
         "Depthmap": 1, "Background": 0, "Depth_range": [float(x) for x in c.depth_range],
         "Resolution": [int(c.width), int(c.height)], "BitDepthColor": int(c.bit_depth_color),
         "BitDepthDepth": int(c.bit_depth_depth), "ColorSpace": "YUV420",
         "DepthColorSpace": "YUV420" if c.depth_color_format == abi.YUV420 else "YUV400",
         "HasInvalidDepth": bool(c.has_invalid_depth)}
    if c.projection == abi.EQUIRECTANGULAR:
        d["Hor_range"] = [float(x) for x in c.hor_range]
        d["Ver_range"] = [float(x) for x in c.ver_range]
    else:
        d["Focal"] = [float(x) for x in c.focal]
        d["Principle_point"] = [float(x) for x in c.principle_point]
    if crop is not None:
        d["Resolution"] = [int(padded[0]), int(padded[1])]
        d["Crop_region"] = [int(v) for v in crop]
        if "Principle_point" in d:
            d["Principle_point"] = [float(c.principle_point[0]) + crop[0], float(c.principle_point[1]) + crop[1]]
    return d


class Camera:
    """A reference Parameters object parsed from an rvsb camera."""

    def __init__(self, cam, crop=None, padded=None):
        self.cam = cam
        self.h = lib().ref_camera_new(json.dumps(camera_dict(cam, crop=crop, padded=padded)).encode())
        if not self.h:
            _check(1)

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.ref_camera_free(self.h)
            self.h = None


def set_precision(p):
    lib().ref_set_precision(float(p))


def set_resize_ties_up(on):
    lib().ref_set_resize_ties_up(1 if on else 0)


def relative_pose(cin, cvirt):
    a, b = Camera(cin), Camera(cvirt)
    R = np.empty(9, np.float32)
    t = np.empty(3, np.float32)
    _check(lib().ref_relative_pose(a.h, b.h, _p(R), _p(t)))
    return R.reshape(3, 3), t


def warp(cin, cvirt, depth):
    a, b = Camera(cin), Camera(cvirt)
    h, w = cin.height, cin.width
    depth = np.ascontiguousarray(depth, np.float32)
    uv = np.empty((h, w, 2), np.float32)
    vd = np.empty((h, w), np.float32)
    wrap = ctypes.c_int(0)
    _check(lib().ref_warp(a.h, b.h, _p(depth), _p(uv), _p(vd), ctypes.byref(wrap)))
    return uv, vd, wrap.value


def raster(color, vdepth, uv, wo, ho, wrap):
    """Returns colour, depth, quality (validity / depth) and validity."""
    h, w = vdepth.shape
    color, vdepth, uv = (np.ascontiguousarray(a, np.float32) for a in (color, vdepth, uv))
    oc = np.empty((ho, wo, 3), np.float32)
    od, oq, ov = (np.empty((ho, wo), np.float32) for _ in range(3))
    _check(lib().ref_raster(_p(color), _p(vdepth), _p(uv), w, h, wo, ho, int(wrap), _p(oc), _p(od), _p(oq), _p(ov)))
    return oc, od, oq, ov


def blend(colors, depths, qualities, validities, exponent, multispectral=None):
    """BlendedViewSimple(exponent), or BlendedViewMultiSpec(low, high) with
    multispectral=(low, high).  Returns colour, quality, depth, validity."""
    n = len(colors)
    ho, wo = qualities[0].shape
    keep = [[np.ascontiguousarray(a, np.float32) for a in arrs] for arrs in (colors, depths, qualities, validities)]
    ptrs = [(_F * n)(*[_p(a) for a in arrs]) for arrs in keep]
    oc = np.empty((ho, wo, 3), np.float32)
    oq, od, ov = (np.empty((ho, wo), np.float32) for _ in range(3))
    ms = multispectral is not None
    low, high = multispectral if ms else (0.0, 0.0)
    _check(lib().ref_blend(n, *ptrs, wo, ho, float(exponent), int(ms), float(low), float(high), _p(oc), _p(oq),
                           _p(od), _p(ov)))
    return oc, oq, od, ov


def inpaint(color, quality):
    ho, wo = quality.shape
    color = np.ascontiguousarray(color, np.float32)
    quality = np.ascontiguousarray(quality, np.float32)
    out = np.empty_like(color)
    _check(lib().ref_inpaint(_p(color), _p(quality), wo, ho, _p(out)))
    return out


def inpaint_sources(hole):
    h, w = hole.shape
    m = np.ascontiguousarray(hole, np.uint8)
    src = np.empty((h, w, 2), np.int32)
    _check(lib().ref_inpaint_sources(_p(m, _U8), w, h, _p(src, _I32)))
    return src


def write_color(color, virt):
    """write_color of a colour image for the virtual camera: (Y, U, V) as
    written to the output file."""
    ho, wo = color.shape[:2]
    color = np.ascontiguousarray(color, np.float32)
    c = Camera(virt)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "out.yuv")
        _check(lib().ref_write_color(_p(color), wo, ho, c.h, path.encode()))
        flat = np.fromfile(path, np.uint16)
    n, q = wo * ho, (wo // 2) * (ho // 2)
    return flat[:n].reshape(ho, wo), flat[n:n + q].reshape(ho // 2, wo // 2), flat[n + q:].reshape(ho // 2, wo // 2)


def synthesize(inputs, colors, depths, virt, exponent, multispectral=None):
    """One synthesized view from decoded inputs through the reference's
    warp, raster, blend and inpainting.  Returns the inpainted colour and the
    blended quality, at the raster size."""
    n = len(inputs)
    cams = [Camera(c) for c in inputs]
    vc = Camera(virt)
    hs = (ctypes.c_void_p * n)(*[c.h for c in cams])
    keep = [[np.ascontiguousarray(a, np.float32) for a in arrs] for arrs in (colors, depths)]
    pc, pd = ((_F * n)(*[_p(a) for a in arrs]) for arrs in keep)
    L = lib()
    # raster size int(0.5 + W * P), the reference's float arithmetic
    P = np.float32(_precision[0])
    wo = int(np.float32(0.5) + np.float32(virt.width) * P)
    ho = int(np.float32(0.5) + np.float32(virt.height) * P)
    oc = np.empty((ho, wo, 3), np.float32)
    oq = np.empty((ho, wo), np.float32)
    ms = multispectral is not None
    low, high = multispectral if ms else (0.0, 0.0)
    _check(L.ref_synthesize(n, hs, pc, pd, vc.h, float(exponent), int(ms), float(low), float(high), _p(oc), _p(oq)))
    return oc, oq


_precision = [1.0]


def set_raster_precision(p):
    """Precision for both the reference (g_rescale) and synthesize()."""
    _precision[0] = float(p)
    set_precision(p)


def load_view(cam, color_path, depth_path, frame, crop=None, padded=None):
    """The reference's loader (read_color / read_depth, image_loading.cpp,
    with its CUDA kernels from process_input_frame.cu): decoded colour
    (H, W, 3) and depth (H, W) of `frame`, H x W the camera's (region's)
    size; with crop / padded (camera_dict) the depth is read at the padded
    size and its first H * W samples returned, as the reference's CPU mode
    copies them (SynthesizedView.cpp:89-94).  Needs a CUDA device."""
    c = Camera(cam, crop, padded)
    color = np.empty((cam.height, cam.width, 3), np.float32)
    depth = np.empty((cam.height, cam.width), np.float32)
    _check(lib().ref_load_view(c.h, color_path.encode(), depth_path.encode(), int(frame), _p(color), _p(depth)))
    return color, depth


def write_aux(kind, depth, mask, virt, crop=None, padded=None):
    """The reference's depth and mask writers (image_writing.cpp:226-302):
    kind "depth" (write_depth), "masked_depth" (write_maskedDepth) or "mask"
    (write_mask) of an output-sized float depth / uint8 mask (nonzero =
    masked) for the virtual camera.  Returns the written file's samples:
    luma plane (uint16, or uint8 for the mask) of the padded size."""
    k = {"depth": 0, "masked_depth": 1, "mask": 2}[kind]
    c = Camera(virt, crop, padded)
    h, w = (mask if depth is None else depth).shape
    dp = np.ascontiguousarray(depth, np.float32) if depth is not None else None
    mp = np.ascontiguousarray(mask, np.uint8) if mask is not None else None
    W, H = padded if padded is not None else (w, h)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "aux.yuv")
        _check(lib().ref_write_aux(k, _p(dp) if dp is not None else None, _p(mp, _U8) if mp is not None else None,
                                   w, h, c.h, path.encode()))
        raw = np.fromfile(path, np.uint8 if kind == "mask" else np.uint16)
    return raw[:W * H].reshape(H, W)
