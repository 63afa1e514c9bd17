"""ctypes mirrors of the plain-C structs in include/rvsb.h.

Only type definitions live here, so the test-side oracle loader can share
them without loading the CUDA library.
"""
import ctypes

RVSB_OK = 0
RVSB_E_ARG = 1
RVSB_E_CONFIG = 2
RVSB_E_IO = 3
RVSB_E_OOM_BUDGET = 4
RVSB_E_CUDA = 5
RVSB_E_TIMEOUT = 6
RVSB_E_UNSUPPORTED = 7
RVSB_E_BUSY = 8
RVSB_E_NOT_FOUND = 9

PERSPECTIVE = 0
EQUIRECTANGULAR = 1
YUV420 = 0
YUV400 = 1


class Camera(ctypes.Structure):
    """rvsb_camera: one camera of an RVS camera-parameter file."""

    _fields_ = [
        ("projection", ctypes.c_int32),
        ("width", ctypes.c_int32),
        ("height", ctypes.c_int32),
        ("bit_depth_color", ctypes.c_int32),
        ("bit_depth_depth", ctypes.c_int32),
        ("depth_color_format", ctypes.c_int32),
        ("has_invalid_depth", ctypes.c_int32),
        ("full_hor_range", ctypes.c_int32),
        ("position", ctypes.c_float * 3),
        ("rotation", ctypes.c_float * 3),
        ("depth_range", ctypes.c_float * 2),
        ("focal", ctypes.c_float * 2),
        ("principle_point", ctypes.c_float * 2),
        ("hor_range", ctypes.c_float * 2),
        ("ver_range", ctypes.c_float * 2),
    ]

    def copy(self):
        c = Camera()
        ctypes.pointer(c)[0] = self
        return c

    def __repr__(self):
        kind = "ERP" if self.projection == EQUIRECTANGULAR else "persp"
        return (f"Camera({kind} {self.width}x{self.height} pos={list(self.position)} "
                f"rot={list(self.rotation)})")


class ViewPlanes(ctypes.Structure):
    """rvsb_view_planes: raw planes of one input view."""

    _fields_ = [
        ("y", ctypes.c_void_p),
        ("u", ctypes.c_void_p),
        ("v", ctypes.c_void_p),
        ("depth", ctypes.c_void_p),
    ]


class Yuv420(ctypes.Structure):
    """rvsb_yuv420: output planes."""

    _fields_ = [
        ("y", ctypes.c_void_p),
        ("u", ctypes.c_void_p),
        ("v", ctypes.c_void_p),
    ]


class SynthParams(ctypes.Structure):
    """rvsb_synth_params."""

    _fields_ = [
        ("blending_factor", ctypes.c_float),
        ("precision", ctypes.c_float),
        ("chroma_rounding", ctypes.c_int32),
        ("blending_method", ctypes.c_int32),
        ("low_freq_factor", ctypes.c_float),
        ("high_freq_factor", ctypes.c_float),
        ("reserved", ctypes.c_int32 * 2),
    ]


class DebugOut(ctypes.Structure):
    """rvsb_debug_out: device pointers for intermediate results."""

    _fields_ = [
        ("warped_uvz", ctypes.c_void_p),
        ("view_color", ctypes.c_void_p),
        ("view_depth", ctypes.c_void_p),
        ("view_validity", ctypes.c_void_p),
        ("blend_color", ctypes.c_void_p),
        ("blend_quality", ctypes.c_void_p),
        ("inpaint_source", ctypes.c_void_p),
    ]


def make_camera(projection=PERSPECTIVE, width=960, height=540, position=(0, 0, 0),
                rotation=(0, 0, 0), depth_range=(0.5, 10.0), focal=(800, 800),
                principle_point=None, hor_range=(-180, 180), ver_range=(-90, 90),
                bit_depth_color=10, bit_depth_depth=16, depth_color_format=YUV420,
                has_invalid_depth=True):
    """Builds a Camera with the JSON defaults of the reference."""
    c = Camera()
    c.projection = projection
    c.width, c.height = width, height
    c.bit_depth_color, c.bit_depth_depth = bit_depth_color, bit_depth_depth
    c.depth_color_format = depth_color_format
    c.has_invalid_depth = 1 if has_invalid_depth else 0
    c.position[:] = [float(x) for x in position]
    c.rotation[:] = [float(x) for x in rotation]
    c.depth_range[:] = [float(x) for x in depth_range]
    c.focal[:] = [float(x) for x in focal]
    if principle_point is None:
        principle_point = (width / 2.0, height / 2.0)
    c.principle_point[:] = [float(x) for x in principle_point]
    c.hor_range[:] = [float(x) for x in hor_range]
    c.ver_range[:] = [float(x) for x in ver_range]
    c.full_hor_range = 1 if (projection == EQUIRECTANGULAR and
                             float(hor_range[0]) == -180.0 and float(hor_range[1]) == 180.0) else 0
    return c


class AuxOut(ctypes.Structure):
    """rvsb_aux_out: device pointers of the auxiliary outputs (NULL = off)."""

    _fields_ = [
        ("mask", ctypes.c_void_p),
        ("masked", Yuv420),
        ("depth", ctypes.c_void_p),
        ("masked_depth", ctypes.c_void_p),
        ("validity_threshold", ctypes.c_float),
        ("reserved", ctypes.c_int32),
    ]
