"""TEST INFRASTRUCTURE ONLY: ctypes loader for the CPU oracle (rvs_oracle.cpp).

Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the
checker.  Nothing in the product library imports this module.
"""
import ctypes
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "rvs-cuda_b200"))
from rvsb import abi  # noqa: E402

LIB_PATH = os.path.join(HERE, "_build", "liborc.so")

_lib = None

_F = ctypes.POINTER(ctypes.c_float)
_U16 = ctypes.POINTER(ctypes.c_uint16)
_I32 = ctypes.POINTER(ctypes.c_int32)


def build():
    """Compiles the oracle with its Makefile (g++ only)."""
    subprocess.check_call(["make", "-s", "-C", HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH) or \
                os.path.getmtime(LIB_PATH) < os.path.getmtime(os.path.join(HERE, "rvs_oracle.cpp")):
            build()
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER(abi.Camera)
        L.orc_set_trig_mode.argtypes = [ctypes.c_int]
        L.orc_set_chroma_round.argtypes = [ctypes.c_int]
        L.orc_set_multispectral.argtypes = [ctypes.c_int, ctypes.c_float, ctypes.c_float]
        L.orc_set_precision.argtypes = [ctypes.c_float]
        L.orc_resize_linear3.argtypes = [_F, ctypes.c_int, ctypes.c_int, _F, ctypes.c_int, ctypes.c_int]
        L.orc_resize_nearest_u8.argtypes = [ctypes.POINTER(ctypes.c_uint8), ctypes.c_int, ctypes.c_int,
                                            ctypes.POINTER(ctypes.c_uint8), ctypes.c_int, ctypes.c_int]
        L.orc_decode_color.argtypes = [_U16, _U16, _U16, ctypes.c_int, ctypes.c_int, ctypes.c_int, _F]
        L.orc_decode_depth.argtypes = [_U16, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                       ctypes.c_float, ctypes.c_int, _F]
        L.orc_rotation_matrix.argtypes = [_F, _F]
        L.orc_relative_pose.argtypes = [P, P, _F, _F]
        L.orc_warp.argtypes = [P, P, _F, _F, _F, ctypes.POINTER(ctypes.c_int)]
        L.orc_raster.argtypes = [_F, _F, _F, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                 ctypes.c_int, _F, _F, _F]
        L.orc_blend.argtypes = [ctypes.c_int, ctypes.POINTER(_F), ctypes.POINTER(_F), ctypes.POINTER(_F),
                                ctypes.c_int, ctypes.c_int, ctypes.c_float, _F, _F]
        L.orc_inpaint.argtypes = [_F, _F, ctypes.c_int, ctypes.c_int, _F, _I32,
                                  ctypes.POINTER(ctypes.c_int)]
        L.orc_write_yuv420.argtypes = [_F, ctypes.c_int, ctypes.c_int, ctypes.c_int, _U16]
        L.orc_synthesize.argtypes = [ctypes.c_int, P, ctypes.POINTER(abi.ViewPlanes), P, ctypes.c_float,
                                     _U16, _F, _F]
        L.orc_synthesize_aux.argtypes = [ctypes.c_int, P, ctypes.POINTER(abi.ViewPlanes), P, ctypes.c_float,
                                         _U16, _F, _F, ctypes.c_float, ctypes.POINTER(ctypes.c_uint8), _U16,
                                         _U16, _U16]
        L.orc_image_pos.argtypes = [P, _F]
        L.orc_unproject.argtypes = [P, _F, _F, _F]
        L.orc_project.argtypes = [P, _F, _F, _F, ctypes.POINTER(ctypes.c_int)]
        L.orc_edge_norm.argtypes = [_F, _F]
        L.orc_edge_norm.restype = ctypes.c_double
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t)


def set_trig_mode(mode):
    lib().orc_set_trig_mode(int(mode))


def set_chroma_round(mode):
    """0: ties to even (OpenCV built with IPP), 1: ties up (without)."""
    lib().orc_set_chroma_round(int(mode))


_precision = np.float32(1.0)


def set_precision(p):
    """'Precision': rasterise at P times the output size, resize when written."""
    global _precision
    _precision = np.float32(p)
    lib().orc_set_precision(float(p))


def raster_size(w, h):
    """(int(0.5 + W * P), int(0.5 + H * P)) in float, as SynthesizedView.cpp:327-329."""
    if _precision == np.float32(1.0):
        return w, h
    return (int(np.float32(0.5) + np.float32(w) * _precision), int(np.float32(0.5) + np.float32(h) * _precision))


def resize_linear3(img, w, h):
    """cv::resize(img, (w, h)) with INTER_LINEAR of an HxWx3 float32 image
    (the output resize of write_color, image_writing.cpp:188-190)."""
    src = np.ascontiguousarray(img, np.float32)
    dst = np.empty((h, w, 3), np.float32)
    lib().orc_resize_linear3(_p(src, _F), src.shape[1], src.shape[0], _p(dst, _F), w, h)
    return dst


def resize_nearest_u8(img, w, h):
    """cv::resize(img, (w, h), INTER_NEAREST) of an HxW uint8 image (the
    validity mask at Precision != 1, Pipeline.cpp:303-308)."""
    src = np.ascontiguousarray(img, np.uint8)
    dst = np.empty((h, w), np.uint8)
    U8 = ctypes.POINTER(ctypes.c_uint8)
    lib().orc_resize_nearest_u8(src.ctypes.data_as(U8), src.shape[1], src.shape[0], dst.ctypes.data_as(U8), w, h)
    return dst


def set_multispectral(on, low=0.0, high=0.0):
    """BlendingMethod Multispectral with the two factors (off: Simple)."""
    lib().orc_set_multispectral(1 if on else 0, float(low), float(high))


def decode_color(y, u, v, bits=10):
    h, w = y.shape
    out = np.empty((h, w, 3), np.float32)
    y, u, v = (np.ascontiguousarray(a, np.uint16) for a in (y, u, v))
    rc = lib().orc_decode_color(_p(y, _U16), _p(u, _U16), _p(v, _U16), w, h, bits, _p(out, _F))
    assert rc == 0, rc
    return out


def decode_depth(d, cam):
    h, w = d.shape
    out = np.empty((h, w), np.float32)
    d = np.ascontiguousarray(d, np.uint16)
    rc = lib().orc_decode_depth(_p(d, _U16), w, h, cam.bit_depth_depth, cam.depth_range[0],
                                cam.depth_range[1], cam.has_invalid_depth, _p(out, _F))
    assert rc == 0, rc
    return out


def rotation_matrix(rot):
    r = np.asarray(rot, np.float32)
    R = np.empty(9, np.float32)
    lib().orc_rotation_matrix(_p(r, _F), _p(R, _F))
    return R.reshape(3, 3)


def relative_pose(cin, cvirt):
    R = np.empty(9, np.float32)
    t = np.empty(3, np.float32)
    lib().orc_relative_pose(ctypes.byref(cin), ctypes.byref(cvirt), _p(R, _F), _p(t, _F))
    return R.reshape(3, 3), t


def warp(cin, cvirt, depth):
    h, w = cin.height, cin.width
    depth = np.ascontiguousarray(depth, np.float32)
    uv = np.empty((h, w, 2), np.float32)
    vd = np.empty((h, w), np.float32)
    wrap = ctypes.c_int(0)
    rc = lib().orc_warp(ctypes.byref(cin), ctypes.byref(cvirt), _p(depth, _F), _p(uv, _F), _p(vd, _F),
                        ctypes.byref(wrap))
    assert rc == 0, rc
    return uv, vd, wrap.value


def raster(color, vdepth, uv, wo, ho, wrap):
    h, w = vdepth.shape
    color = np.ascontiguousarray(color, np.float32)
    vdepth = np.ascontiguousarray(vdepth, np.float32)
    uv = np.ascontiguousarray(uv, np.float32)
    oc = np.empty((ho, wo, 3), np.float32)
    od = np.empty((ho, wo), np.float32)
    ov = np.empty((ho, wo), np.float32)
    rc = lib().orc_raster(_p(color, _F), _p(vdepth, _F), _p(uv, _F), w, h, wo, ho, int(wrap), _p(oc, _F),
                          _p(od, _F), _p(ov, _F))
    assert rc == 0, rc
    return oc, od, ov


def blend(colors, qualities, depths, exponent):
    n = len(colors)
    ho, wo = qualities[0].shape
    colors = [np.ascontiguousarray(c, np.float32) for c in colors]
    qualities = [np.ascontiguousarray(q, np.float32) for q in qualities]
    depths = [np.ascontiguousarray(d, np.float32) for d in depths]
    pc = (_F * n)(*[_p(c, _F) for c in colors])
    pq = (_F * n)(*[_p(q, _F) for q in qualities])
    pd = (_F * n)(*[_p(d, _F) for d in depths])
    oc = np.empty((ho, wo, 3), np.float32)
    oq = np.empty((ho, wo), np.float32)
    rc = lib().orc_blend(n, pc, pq, pd, wo, ho, float(exponent), _p(oc, _F), _p(oq, _F))
    assert rc == 0, rc
    return oc, oq


def inpaint(color, quality):
    ho, wo = quality.shape
    color = np.ascontiguousarray(color, np.float32)
    quality = np.ascontiguousarray(quality, np.float32)
    out = np.empty_like(color)
    src = np.empty((ho, wo, 2), np.int32)
    sweeps = ctypes.c_int(0)
    rc = lib().orc_inpaint(_p(color, _F), _p(quality, _F), wo, ho, _p(out, _F), _p(src, _I32),
                           ctypes.byref(sweeps))
    assert rc == 0, rc
    return out, src, sweeps.value


def write_yuv420(color, bits=10):
    ho, wo = color.shape[:2]
    color = np.ascontiguousarray(color, np.float32)
    out = np.empty(wo * ho * 3 // 2, np.uint16)
    rc = lib().orc_write_yuv420(_p(color, _F), wo, ho, bits, _p(out, _U16))
    assert rc == 0, rc
    return split_yuv420(out, wo, ho)


def split_yuv420(flat, wo, ho):
    n = wo * ho
    c = (wo // 2) * (ho // 2)
    return (flat[:n].reshape(ho, wo), flat[n:n + c].reshape(ho // 2, wo // 2),
            flat[n + c:n + 2 * c].reshape(ho // 2, wo // 2))


def synthesize(inputs, planes, virt, exponent, want_intermediate=False):
    """Full CPU synthesis of one view.  planes: list of (Y, U, V, D) arrays.
    Returns (Y, U, V) and optionally (blended quality, blended colour)."""
    n = len(inputs)
    cams = (abi.Camera * n)(*inputs)
    keep = []
    vp = (abi.ViewPlanes * n)()
    for i, (y, u, v, d) in enumerate(planes):
        arrs = [np.ascontiguousarray(a, np.uint16) for a in (y, u, v, d)]
        keep.append(arrs)
        vp[i].y, vp[i].u, vp[i].v, vp[i].depth = (a.ctypes.data for a in arrs)
    wo, ho = virt.width, virt.height
    out = np.empty(wo * ho * 3 // 2, np.uint16)
    rw, rh = raster_size(wo, ho)
    q = np.empty((rh, rw), np.float32) if want_intermediate else None
    c = np.empty((rh, rw, 3), np.float32) if want_intermediate else None
    rc = lib().orc_synthesize(n, cams, vp, ctypes.byref(virt), float(exponent), _p(out, _U16),
                              _p(q, _F) if q is not None else None,
                              _p(c, _F) if c is not None else None)
    assert rc == 0, rc
    yuv = split_yuv420(out, wo, ho)
    if want_intermediate:
        return yuv, q, c
    return yuv


def synthesize_aux(inputs, planes, virt, exponent, threshold=5000.0, masked=True):
    """Synthesis with the auxiliary outputs of Pipeline.cpp:303-336.  Returns
    a dict: yuv, mask (uint8), masked_yuv (masked=True only), depth and
    masked_depth (uint16), all at the virtual camera's size."""
    n = len(inputs)
    cams = (abi.Camera * n)(*inputs)
    keep = []
    vp = (abi.ViewPlanes * n)()
    for i, (y, u, v, d) in enumerate(planes):
        arrs = [np.ascontiguousarray(a, np.uint16) for a in (y, u, v, d)]
        keep.append(arrs)
        vp[i].y, vp[i].u, vp[i].v, vp[i].depth = (a.ctypes.data for a in arrs)
    wo, ho = virt.width, virt.height
    out = np.empty(wo * ho * 3 // 2, np.uint16)
    masked_out = np.empty(wo * ho * 3 // 2, np.uint16)
    mask = np.empty((ho, wo), np.uint8)
    depth = np.empty((ho, wo), np.uint16)
    mdepth = np.empty((ho, wo), np.uint16)
    rc = lib().orc_synthesize_aux(n, cams, vp, ctypes.byref(virt), float(exponent), _p(out, _U16), None, None,
                                  float(threshold), mask.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)),
                                  _p(masked_out, _U16) if masked else None, _p(depth, _U16), _p(mdepth, _U16))
    assert rc == 0, rc
    r = {"yuv": split_yuv420(out, wo, ho), "mask": mask, "depth": depth, "masked_depth": mdepth}
    if masked:
        r["masked_yuv"] = split_yuv420(masked_out, wo, ho)
    return r


def image_pos(cam):
    uv = np.empty((cam.height, cam.width, 2), np.float32)
    assert lib().orc_image_pos(ctypes.byref(cam), _p(uv, _F)) == 0
    return uv


def unproject(cam, uv, depth):
    uv = np.ascontiguousarray(uv, np.float32)
    depth = np.ascontiguousarray(depth, np.float32)
    xyz = np.empty((cam.height, cam.width, 3), np.float32)
    assert lib().orc_unproject(ctypes.byref(cam), _p(uv, _F), _p(depth, _F), _p(xyz, _F)) == 0
    return xyz


def project(cam, xyz):
    xyz = np.ascontiguousarray(xyz, np.float32)
    uv = np.empty((cam.height, cam.width, 2), np.float32)
    d = np.empty((cam.height, cam.width), np.float32)
    wrap = ctypes.c_int(0)
    assert lib().orc_project(ctypes.byref(cam), _p(xyz, _F), _p(uv, _F), _p(d, _F), ctypes.byref(wrap)) == 0
    return uv, d, wrap.value


def edge_norm(a, b):
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    return lib().orc_edge_norm(_p(a, _F), _p(b, _F))
