"""Python binding (ctypes) of the B200 RVS synthesis backend, librvsb.so.

The library is the product: every call goes through the C ABI declared in
include/rvsb.h.  Loading fails loudly when the library is missing; there is
no fallback implementation.

Device buffers are passed as raw pointers (e.g. torch tensors' data_ptr()),
streams as cudaStream_t handles (torch.cuda.Stream.cuda_stream).
"""
import ctypes
import os

from .abi import (AuxOut, Camera, DebugOut, SynthParams, ViewPlanes, Yuv420, make_camera, PERSPECTIVE,
                  EQUIRECTANGULAR, YUV420, YUV400, RVSB_OK)
from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(HERE), "lib", "librvsb.so")

# Every entry point include/rvsb.h declares.
EXPORTED = [
    "rvsb_create", "rvsb_destroy", "rvsb_last_error", "rvsb_status_string", "rvsb_memory_in_use",
    "rvsb_camera_from_json", "rvsb_config_load", "rvsb_config_free", "rvsb_config_num_inputs",
    "rvsb_config_num_virtual", "rvsb_config_input_camera", "rvsb_config_virtual_camera",
    "rvsb_config_texture_path", "rvsb_config_depth_path", "rvsb_config_output_path", "rvsb_config_frames",
    "rvsb_config_synth_params", "rvsb_config_virtual_camera_at", "rvsb_relative_pose", "rvsb_scene_create",
    "rvsb_scene_destroy", "rvsb_scene_upload", "rvsb_synthesize", "rvsb_synthesize_host",
    "rvsb_synthesize_debug", "rvsb_synthesize_frame", "rvsb_scene_last_launch_count", "rvsb_scene_set_profiling",
    "rvsb_scene_stage_times", "rvsb_stage_name", "rvsb_inpaint_sources_noalloc",
    "rvsb_batch_create", "rvsb_batch_destroy", "rvsb_batch_reserve", "rvsb_batch_set_graphs",
    "rvsb_synthesize_batch", "rvsb_batch_last_launch_count", "rvsb_batch_set_profiling", "rvsb_batch_stage_times",
    "rvsb_server_create", "rvsb_server_add_scene", "rvsb_server_reserve", "rvsb_server_submit", "rvsb_server_poll",
    "rvsb_server_drain", "rvsb_server_clock", "rvsb_server_destroy",
    "rvsb_batch_set_autotune", "rvsb_batch_set_raster_variant", "rvsb_batch_last_raster_variant",
    "rvsb_scene_set_autotune", "rvsb_scene_set_raster_variant", "rvsb_synthesize_aux", "rvsb_config_output_file", "rvsb_config_validity_threshold",
    "rvsb_config_virtual_crop", "rvsb_config_input_crop", "rvsb_host_stream_create", "rvsb_host_stream_destroy", "rvsb_host_stream_submit",
    "rvsb_host_stream_wait", "rvsb_host_stream_join",
]

OUT_COLOR, OUT_MASKED_COLOR, OUT_MASK, OUT_DEPTH, OUT_MASKED_DEPTH = range(5)

RASTER_VARIANTS = 8

STAGES = ["warp", "bin", "raster", "inpaint", "total"]

_lib = None


class RvsbError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"rvsb status {status}: {msg}")
        self.status = status


def load():
    """Loads librvsb.so (built by rvs-cuda_b200/build.py)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"native library missing: {LIB_PATH} (run rvs-cuda_b200/build.py)")
    L = ctypes.CDLL(LIB_PATH)
    c_p = ctypes.c_void_p
    P = ctypes.POINTER
    L.rvsb_create.argtypes = [ctypes.c_int, ctypes.c_size_t, P(c_p)]
    L.rvsb_destroy.argtypes = [c_p]
    L.rvsb_destroy.restype = None
    L.rvsb_last_error.argtypes = [c_p]
    L.rvsb_last_error.restype = ctypes.c_char_p
    L.rvsb_status_string.argtypes = [ctypes.c_int]
    L.rvsb_status_string.restype = ctypes.c_char_p
    L.rvsb_memory_in_use.argtypes = [c_p]
    L.rvsb_memory_in_use.restype = ctypes.c_size_t
    L.rvsb_camera_from_json.argtypes = [ctypes.c_char_p, P(Camera), ctypes.c_char_p, ctypes.c_size_t]
    L.rvsb_config_load.argtypes = [ctypes.c_char_p, P(c_p), ctypes.c_char_p, ctypes.c_size_t]
    L.rvsb_config_free.argtypes = [c_p]
    L.rvsb_config_free.restype = None
    L.rvsb_config_num_inputs.argtypes = [c_p]
    L.rvsb_config_num_virtual.argtypes = [c_p]
    L.rvsb_config_input_camera.argtypes = [c_p, ctypes.c_int, P(Camera)]
    L.rvsb_config_virtual_camera.argtypes = [c_p, ctypes.c_int, P(Camera)]
    for f in ("rvsb_config_texture_path", "rvsb_config_depth_path", "rvsb_config_output_path"):
        getattr(L, f).argtypes = [c_p, ctypes.c_int]
        getattr(L, f).restype = ctypes.c_char_p
    L.rvsb_config_frames.argtypes = [c_p, P(ctypes.c_int), P(ctypes.c_int), P(ctypes.c_int)]
    L.rvsb_config_frames.restype = None
    L.rvsb_config_synth_params.argtypes = [c_p, P(SynthParams)]
    L.rvsb_config_synth_params.restype = None
    L.rvsb_config_virtual_camera_at.argtypes = [c_p, ctypes.c_int, ctypes.c_int, P(Camera)]
    L.rvsb_config_virtual_crop.argtypes = [c_p, ctypes.c_int, P(ctypes.c_int32), P(ctypes.c_int32)]
    L.rvsb_config_input_crop.argtypes = [c_p, ctypes.c_int, P(ctypes.c_int32), P(ctypes.c_int32)]
    L.rvsb_relative_pose.argtypes = [P(Camera), P(Camera), P(ctypes.c_float), P(ctypes.c_float)]
    L.rvsb_scene_create.argtypes = [c_p, P(Camera), ctypes.c_int, P(c_p)]
    L.rvsb_scene_destroy.argtypes = [c_p]
    L.rvsb_scene_destroy.restype = None
    L.rvsb_scene_upload.argtypes = [c_p, ctypes.c_int, P(ViewPlanes), ctypes.c_int, c_p]
    L.rvsb_synthesize.argtypes = [c_p, P(Camera), P(SynthParams), P(Yuv420), c_p]
    L.rvsb_synthesize_host.argtypes = [c_p, P(Camera), ctypes.c_int, P(ViewPlanes), P(Camera),
                                       P(SynthParams), P(Yuv420), c_p]
    L.rvsb_host_stream_create.argtypes = [c_p, P(Camera), ctypes.c_int, P(c_p)]
    L.rvsb_host_stream_destroy.argtypes = [c_p]
    L.rvsb_host_stream_destroy.restype = None
    L.rvsb_host_stream_submit.argtypes = [c_p, P(ViewPlanes), P(Camera), P(SynthParams), P(Yuv420), c_p,
                                          P(ctypes.c_uint64)]
    L.rvsb_host_stream_wait.argtypes = [c_p, ctypes.c_uint64]
    L.rvsb_host_stream_join.argtypes = [c_p, c_p]
    L.rvsb_synthesize_debug.argtypes = [c_p, P(Camera), P(SynthParams), P(Yuv420), P(DebugOut), c_p]
    L.rvsb_synthesize_frame.argtypes = [c_p, P(ViewPlanes), P(Camera), P(SynthParams), P(Yuv420), c_p]
    L.rvsb_scene_last_launch_count.argtypes = [c_p]
    L.rvsb_scene_set_profiling.argtypes = [c_p, ctypes.c_int]
    L.rvsb_scene_stage_times.argtypes = [c_p, P(ctypes.c_float), ctypes.c_int]
    L.rvsb_stage_name.argtypes = [ctypes.c_int]
    L.rvsb_stage_name.restype = ctypes.c_char_p
    L.rvsb_batch_create.argtypes = [c_p, ctypes.c_int, P(c_p)]
    L.rvsb_batch_destroy.argtypes = [c_p]
    L.rvsb_batch_destroy.restype = None
    L.rvsb_batch_reserve.argtypes = [c_p, ctypes.c_int, ctypes.c_int]
    L.rvsb_batch_set_graphs.argtypes = [c_p, ctypes.c_int]
    L.rvsb_synthesize_batch.argtypes = [c_p, P(Camera), ctypes.c_int, P(SynthParams), P(Yuv420), c_p]
    L.rvsb_batch_last_launch_count.argtypes = [c_p]
    L.rvsb_batch_set_profiling.argtypes = [c_p, ctypes.c_int]
    L.rvsb_batch_stage_times.argtypes = [c_p, P(ctypes.c_float), ctypes.c_int]
    L.rvsb_synthesize_aux.argtypes = [c_p, P(Camera), P(SynthParams), P(Yuv420), P(AuxOut), c_p]
    L.rvsb_config_output_file.argtypes = [c_p, ctypes.c_int, ctypes.c_int]
    L.rvsb_config_output_file.restype = ctypes.c_char_p
    L.rvsb_config_validity_threshold.argtypes = [c_p]
    L.rvsb_config_validity_threshold.restype = ctypes.c_float
    L.rvsb_batch_set_autotune.argtypes = [c_p, ctypes.c_int]
    L.rvsb_batch_set_raster_variant.argtypes = [c_p, ctypes.c_int]
    L.rvsb_batch_last_raster_variant.argtypes = [c_p]
    L.rvsb_scene_set_autotune.argtypes = [c_p, ctypes.c_int]
    L.rvsb_scene_set_raster_variant.argtypes = [c_p, ctypes.c_int]
    L.rvsb_server_create.argtypes = [c_p, ctypes.c_int, ctypes.c_int, ctypes.c_size_t, P(c_p)]
    L.rvsb_server_add_scene.argtypes = [c_p, c_p, P(ctypes.c_int)]
    L.rvsb_server_reserve.argtypes = [c_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.rvsb_server_submit.argtypes = [c_p, ctypes.c_int, P(Camera), P(SynthParams), P(Yuv420), P(ctypes.c_uint64)]
    L.rvsb_server_poll.argtypes = [c_p, P(RequestResult), ctypes.c_int]
    L.rvsb_server_drain.argtypes = [c_p, ctypes.c_int]
    L.rvsb_server_clock.argtypes = [c_p]
    L.rvsb_server_clock.restype = ctypes.c_double
    L.rvsb_server_destroy.argtypes = [c_p]
    L.rvsb_server_destroy.restype = None
    L.rvsb_inpaint_sources_noalloc.argtypes = [c_p, ctypes.c_int, ctypes.c_int, c_p, c_p, ctypes.c_char_p,
                                               ctypes.c_size_t]
    _lib = L
    return L


def status_string(status):
    return load().rvsb_status_string(status).decode()


CHROMA_TIES_EVEN = 0  # output chroma rounding of OpenCV built with IPP
CHROMA_TIES_UP = 1    # ... and without it


BLEND_SIMPLE, BLEND_MULTISPECTRAL = 0, 1


def params(blending_factor=5.0, precision=1.0, chroma_rounding=CHROMA_TIES_EVEN, multispectral=None):
    """Synthesis options; multispectral=(low, high) selects BlendingMethod
    Multispectral with those factors."""
    p = SynthParams()
    p.blending_factor = blending_factor
    p.precision = precision
    p.chroma_rounding = chroma_rounding
    if multispectral is not None:
        p.blending_method = BLEND_MULTISPECTRAL
        p.low_freq_factor, p.high_freq_factor = multispectral
    return p


class Context:
    """rvsb_context: one CUDA device and an HBM budget."""

    def __init__(self, device=0, hbm_budget=0):
        self.lib = load()
        h = ctypes.c_void_p()
        st = self.lib.rvsb_create(int(device), int(hbm_budget), ctypes.byref(h))
        if st != RVSB_OK:
            raise RvsbError(st, "rvsb_create failed: " + status_string(st))
        self.h = h

    def check(self, st):
        if st != RVSB_OK:
            raise RvsbError(st, self.last_error())
        return st

    def last_error(self):
        return self.lib.rvsb_last_error(self.h).decode()

    def memory_in_use(self):
        return self.lib.rvsb_memory_in_use(self.h)

    def close(self):
        if self.h:
            self.lib.rvsb_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def synthesize_host(self, cams, host_planes, virt, p, out_planes, stream=None):
        """Plain per-view call with host buffers (numpy or pinned torch)."""
        n = len(cams)
        arr = (Camera * n)(*cams)
        vp = (ViewPlanes * n)()
        for i, planes in enumerate(host_planes):
            vp[i].y, vp[i].u, vp[i].v, vp[i].depth = (_ptr(a) for a in planes)
        out = Yuv420(*(_ptr(a) for a in out_planes))
        return self.check(self.lib.rvsb_synthesize_host(self.h, arr, n, vp, ctypes.byref(virt),
                                                        ctypes.byref(p), ctypes.byref(out),
                                                        _stream(stream)))


class HostStream:
    """rvsb_host_stream: frames with host buffers, uploads, synthesis and
    downloads of consecutive frames overlapped (three frames in flight)."""

    def __init__(self, ctx, cams):
        self.ctx = ctx
        self.cams = list(cams)
        n = len(self.cams)
        h = ctypes.c_void_p()
        ctx.check(ctx.lib.rvsb_host_stream_create(ctx.h, (Camera * n)(*self.cams), n, ctypes.byref(h)))
        self.h = h

    def submit(self, host_planes, virt, p, out_planes, stream=None):
        """Enqueues one frame; returns its ticket.  The buffers must stay
        untouched until wait(ticket)."""
        n = len(self.cams)
        vp = (ViewPlanes * n)()
        for i, planes in enumerate(host_planes):
            vp[i].y, vp[i].u, vp[i].v, vp[i].depth = (_ptr(a) for a in planes)
        out = Yuv420(*(_ptr(a) for a in out_planes))
        t = ctypes.c_uint64()
        self.ctx.check(self.ctx.lib.rvsb_host_stream_submit(self.h, vp, ctypes.byref(virt), ctypes.byref(p),
                                                            ctypes.byref(out), _stream(stream), ctypes.byref(t)))
        return t.value

    def wait(self, ticket):
        return self.ctx.check(self.ctx.lib.rvsb_host_stream_wait(self.h, ctypes.c_uint64(ticket)))

    def join(self, stream=None):
        return self.ctx.check(self.ctx.lib.rvsb_host_stream_join(self.h, _stream(stream)))

    def close(self):
        if self.h:
            self.ctx.lib.rvsb_host_stream_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Scene:
    """rvsb_scene: input views resident in device memory."""

    def __init__(self, ctx, cams):
        self.ctx = ctx
        self.cams = list(cams)
        n = len(self.cams)
        h = ctypes.c_void_p()
        ctx.check(ctx.lib.rvsb_scene_create(ctx.h, (Camera * n)(*self.cams), n, ctypes.byref(h)))
        self.h = h

    def upload(self, view, planes, on_device, stream=None):
        vp = ViewPlanes(*(_ptr(a) for a in planes))
        return self.ctx.check(self.ctx.lib.rvsb_scene_upload(self.h, int(view), ctypes.byref(vp),
                                                             1 if on_device else 0, _stream(stream)))

    def synthesize(self, virt, p, out_planes, stream=None):
        out = Yuv420(*(_ptr(a) for a in out_planes))
        return self.ctx.check(self.ctx.lib.rvsb_synthesize(self.h, ctypes.byref(virt), ctypes.byref(p),
                                                           ctypes.byref(out), _stream(stream)))

    def synthesize_aux(self, virt, p, out_planes, mask=None, masked=None, depth=None, masked_depth=None,
                       validity_threshold=5000.0, stream=None):
        """rvsb_synthesize_aux: the output planes plus the auxiliary outputs
        (device buffers; any may be None)."""
        out = Yuv420(*(_ptr(a) for a in out_planes))
        aux = AuxOut()
        aux.mask = _ptr(mask)
        if masked is not None:
            aux.masked = Yuv420(*(_ptr(a) for a in masked))
        aux.depth = _ptr(depth)
        aux.masked_depth = _ptr(masked_depth)
        aux.validity_threshold = validity_threshold
        return self.ctx.check(self.ctx.lib.rvsb_synthesize_aux(self.h, ctypes.byref(virt), ctypes.byref(p),
                                                               ctypes.byref(out), ctypes.byref(aux), _stream(stream)))

    def synthesize_frame(self, device_planes, virt, p, out_planes, stream=None):
        """Per-frame call with raw planes in device memory (no copies)."""
        n = len(self.cams)
        vp = (ViewPlanes * n)()
        for i, planes in enumerate(device_planes):
            vp[i].y, vp[i].u, vp[i].v, vp[i].depth = (_ptr(a) for a in planes)
        out = Yuv420(*(_ptr(a) for a in out_planes))
        return self.ctx.check(self.ctx.lib.rvsb_synthesize_frame(self.h, vp, ctypes.byref(virt), ctypes.byref(p),
                                                                 ctypes.byref(out), _stream(stream)))

    def synthesize_debug(self, virt, p, out_planes, dbg, stream=None):
        out = Yuv420(*(_ptr(a) for a in out_planes))
        d = DebugOut(*(_ptr(dbg.get(k)) for k in ("warped_uvz", "view_color", "view_depth",
                                                   "view_validity", "blend_color", "blend_quality",
                                                   "inpaint_source")))
        return self.ctx.check(self.ctx.lib.rvsb_synthesize_debug(self.h, ctypes.byref(virt), ctypes.byref(p),
                                                                 ctypes.byref(out), ctypes.byref(d),
                                                                 _stream(stream)))

    def last_launch_count(self):
        return self.ctx.lib.rvsb_scene_last_launch_count(self.h)

    def set_profiling(self, on=True):
        return self.ctx.check(self.ctx.lib.rvsb_scene_set_profiling(self.h, 1 if on else 0))

    def set_autotune(self, on=True):
        return self.ctx.check(self.ctx.lib.rvsb_scene_set_autotune(self.h, 1 if on else 0))

    def set_raster_variant(self, v):
        """Pins the raster variant of this scene's calls (-1: default or tuned)."""
        return self.ctx.check(self.ctx.lib.rvsb_scene_set_raster_variant(self.h, int(v)))

    def stage_times(self):
        """{stage: ms} of the last profiled synthesis (stream must be complete)."""
        buf = (ctypes.c_float * len(STAGES))()
        n = self.ctx.lib.rvsb_scene_stage_times(self.h, buf, len(STAGES))
        if n < 0:
            raise RvsbError(-1, "no profiled synthesis")
        return {STAGES[i]: buf[i] for i in range(n)}

    def close(self):
        if self.h:
            self.ctx.lib.rvsb_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """rvsb_batch: up to `slots` virtual views of one scene per launch group."""

    def __init__(self, scene, slots, graphs=False):
        self.scene = scene
        self.ctx = scene.ctx
        h = ctypes.c_void_p()
        self.ctx.check(self.ctx.lib.rvsb_batch_create(scene.h, int(slots), ctypes.byref(h)))
        self.h = h
        self.slots = slots
        if graphs:
            self.set_graphs(True)

    def reserve(self, max_width, max_height):
        return self.ctx.check(self.ctx.lib.rvsb_batch_reserve(self.h, int(max_width), int(max_height)))

    def set_graphs(self, on=True):
        return self.ctx.check(self.ctx.lib.rvsb_batch_set_graphs(self.h, 1 if on else 0))

    def set_profiling(self, on=True):
        return self.ctx.check(self.ctx.lib.rvsb_batch_set_profiling(self.h, 1 if on else 0))

    def set_autotune(self, on=True):
        return self.ctx.check(self.ctx.lib.rvsb_batch_set_autotune(self.h, 1 if on else 0))

    def set_raster_variant(self, v):
        return self.ctx.check(self.ctx.lib.rvsb_batch_set_raster_variant(self.h, int(v)))

    def last_raster_variant(self):
        return self.ctx.lib.rvsb_batch_last_raster_variant(self.h)

    def stage_times(self):
        buf = (ctypes.c_float * len(STAGES))()
        n = self.ctx.lib.rvsb_batch_stage_times(self.h, buf, len(STAGES))
        if n < 0:
            raise RvsbError(-1, "no profiled batch")
        return {STAGES[i]: buf[i] for i in range(n)}

    def last_launch_count(self):
        return self.ctx.lib.rvsb_batch_last_launch_count(self.h)

    def synthesize(self, virts, p, outs, stream=None):
        """virts: cameras; outs: one (y, u, v) device triple per camera."""
        n = len(virts)
        cams = (Camera * n)(*virts)
        ys = (Yuv420 * n)(*[Yuv420(*(_ptr(a) for a in o)) for o in outs])
        return self.ctx.check(self.ctx.lib.rvsb_synthesize_batch(self.h, cams, n, ctypes.byref(p), ys,
                                                                 _stream(stream)))

    def close(self):
        if self.h:
            self.ctx.lib.rvsb_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class RequestResult(ctypes.Structure):
    """rvsb_request_result."""

    _fields_ = [("id", ctypes.c_uint64), ("status", ctypes.c_int32), ("batch_size", ctypes.c_int32),
                ("submit_s", ctypes.c_double), ("start_s", ctypes.c_double), ("done_s", ctypes.c_double)]


class Server:
    """rvsb_server: requests on resident scenes with continuous batching."""

    def __init__(self, ctx, lanes=4, max_batch=4, hbm_budget=0):
        self.ctx = ctx
        self.lib = ctx.lib
        h = ctypes.c_void_p()
        ctx.check(self.lib.rvsb_server_create(ctx.h, int(lanes), int(max_batch), int(hbm_budget), ctypes.byref(h)))
        self.h = h
        self._keep = {}

    def add_scene(self, scene):
        sid = ctypes.c_int()
        self.ctx.check(self.lib.rvsb_server_add_scene(self.h, scene.h, ctypes.byref(sid)))
        return sid.value

    def reserve(self, scene_id, max_width, max_height):
        return self.ctx.check(self.lib.rvsb_server_reserve(self.h, int(scene_id), int(max_width), int(max_height)))

    def submit(self, scene_id, virt, p, out_planes):
        out = Yuv420(*(_ptr(a) for a in out_planes))
        rid = ctypes.c_uint64()
        self.ctx.check(self.lib.rvsb_server_submit(self.h, int(scene_id), ctypes.byref(virt), ctypes.byref(p),
                                                   ctypes.byref(out), ctypes.byref(rid)))
        return rid.value

    def poll(self, max_results=4096):
        buf = (RequestResult * max_results)()
        n = self.lib.rvsb_server_poll(self.h, buf, max_results)
        return [(r.id, r.status, r.batch_size, r.submit_s, r.start_s, r.done_s) for r in buf[:n]]

    def drain(self, timeout_ms=60000):
        return self.ctx.check(self.lib.rvsb_server_drain(self.h, int(timeout_ms)))

    def clock(self):
        return self.lib.rvsb_server_clock(self.h)

    def close(self):
        if self.h:
            self.lib.rvsb_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _ptr(a):
    """Raw address of a numpy array, torch tensor or int (None -> NULL)."""
    if a is None:
        return None
    if isinstance(a, int):
        return a
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    if hasattr(a, "ctypes"):
        return a.ctypes.data
    raise TypeError(f"cannot take the address of {type(a)}")


def _stream(s):
    if s is None:
        return None
    if isinstance(s, int):
        return s
    return s.cuda_stream


def inpaint_sources_noalloc(holes, width, height, sources, stream=None):
    """rvsb_inpaint_sources_noalloc: device hole mask (uint8, nonzero =
    hole) -> device (x, y) int32 source per pixel, without allocation."""
    L = load()
    err = ctypes.create_string_buffer(512)
    st = L.rvsb_inpaint_sources_noalloc(_ptr(holes), int(width), int(height), _ptr(sources), _stream(stream),
                                        err, 512)
    if st != RVSB_OK:
        raise RvsbError(st, err.value.decode())


def relative_pose(cin, cvirt):
    L = load()
    R = (ctypes.c_float * 9)()
    t = (ctypes.c_float * 3)()
    L.rvsb_relative_pose(ctypes.byref(cin), ctypes.byref(cvirt), R, t)
    return list(R), list(t)


def camera_from_json(text):
    L = load()
    c = Camera()
    err = ctypes.create_string_buffer(1024)
    st = L.rvsb_camera_from_json(text.encode(), ctypes.byref(c), err, 1024)
    if st != RVSB_OK:
        raise RvsbError(st, err.value.decode())
    return c


def crop_depth_plane(padded_luma, width, height):
    """The depth plane of an input camera with Crop_region: the reference
    decodes the padded depth frame and takes its first width * height
    samples in memory order as the region-sized map (image_loading.cpp:149,
    SynthesizedView.cpp:89-94).  padded_luma: the padded frame's luma plane
    (any shape, row-major)."""
    import numpy as np
    flat = np.ascontiguousarray(padded_luma).reshape(-1)
    if flat.size < width * height:
        raise ValueError("the padded depth frame is smaller than the region")
    return flat[:width * height].reshape(height, width)


class Config:
    """rvsb_config: an RVS configuration file and its camera files."""

    def __init__(self, path):
        self.lib = load()
        h = ctypes.c_void_p()
        err = ctypes.create_string_buffer(1024)
        st = self.lib.rvsb_config_load(str(path).encode(), ctypes.byref(h), err, 1024)
        if st != RVSB_OK:
            raise RvsbError(st, err.value.decode())
        self.h = h

    def inputs(self):
        n = self.lib.rvsb_config_num_inputs(self.h)
        out = []
        for i in range(n):
            c = Camera()
            self.lib.rvsb_config_input_camera(self.h, i, ctypes.byref(c))
            out.append(c)
        return out

    def virtual(self, i=0, frame=None):
        c = Camera()
        if frame is None:
            st = self.lib.rvsb_config_virtual_camera(self.h, i, ctypes.byref(c))
        else:
            st = self.lib.rvsb_config_virtual_camera_at(self.h, i, frame, ctypes.byref(c))
        if st != RVSB_OK:
            raise RvsbError(st, "no such virtual camera / frame")
        return c

    def virtual_crop(self, i=0):
        """((x, y, width, height), (padded width, padded height)) of virtual camera i."""
        r = (ctypes.c_int32 * 4)()
        s = (ctypes.c_int32 * 2)()
        st = self.lib.rvsb_config_virtual_crop(self.h, i, r, s)
        if st != RVSB_OK:
            raise RvsbError(st, "no such virtual camera")
        return tuple(r), tuple(s)

    def input_crop(self, i=0):
        """((x, y, width, height), (padded width, padded height)) of input
        camera i.  The view's depth plane is the first width * height
        samples of the padded depth frame's luma (crop_depth_plane)."""
        r = (ctypes.c_int32 * 4)()
        s = (ctypes.c_int32 * 2)()
        st = self.lib.rvsb_config_input_crop(self.h, i, r, s)
        if st != RVSB_OK:
            raise RvsbError(st, "no such input camera")
        return tuple(r), tuple(s)

    def frames(self):
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self.lib.rvsb_config_frames(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
        return a.value, b.value, c.value

    def synth_params(self):
        p = SynthParams()
        self.lib.rvsb_config_synth_params(self.h, ctypes.byref(p))
        return p

    def paths(self, i):
        f = lambda g: (g(self.h, i) or b"").decode()
        return f(self.lib.rvsb_config_texture_path), f(self.lib.rvsb_config_depth_path)

    def output_file(self, kind, i=0):
        r = self.lib.rvsb_config_output_file(self.h, int(kind), i)
        return r.decode() if r else None

    def validity_threshold(self):
        return self.lib.rvsb_config_validity_threshold(self.h)

    def output_path(self, i=0):
        r = self.lib.rvsb_config_output_path(self.h, i)
        return r.decode() if r else None

    def close(self):
        if self.h:
            self.lib.rvsb_config_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
