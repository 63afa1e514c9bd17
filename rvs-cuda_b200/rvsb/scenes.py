"""Seeded synthetic scenes in the reference's input formats.

The MPEG content the reference was measured on (ClassroomVideo, Museum,
Chess) is not available, so every workload here is a seeded synthetic scene
with the same file formats: 10-bit YUV420 texture in 16-bit little-endian
samples and a 16-bit normalised-disparity depth map (the inverse of the
decode in rvs_cuda_lib/src/process_input_frame.cu:369-376).

Scenes are ray cast analytically per camera pixel (closest hit of planes,
spheres and boxes); a miss takes the far plane.  Texture is 3-D value noise
evaluated at the hit point (so it agrees between views) plus flat-colour
patches.  Cameras follow the reference axes: x forward, y left, z up,
rotation = (yaw, pitch, roll) in degrees (rvs/src/Parameters.cpp:67-97).

Workload names follow the five benchmark configurations:
  plain_small   2 perspective 960x540 inputs -> 1 view at the midpoint
  plain_1080p   4 perspective 1920x1080 inputs on a 2x2 grid -> 1 view
  batched_erp   4 ERP 4096x2048 inputs -> 1080p perspective trajectory
  batched_mixed 11 perspective 2048x1088 inputs -> mixed-size targets
"""
import math
import os

import numpy as np

from . import abi

def rotation_matrix(rot_deg):
    """Rz(yaw) * Ry(pitch) * Rx(roll), float64 (camera -> world)."""
    a, b, c = (math.radians(float(x)) for x in rot_deg)
    rz = np.array([[math.cos(a), -math.sin(a), 0], [math.sin(a), math.cos(a), 0], [0, 0, 1]])
    ry = np.array([[math.cos(b), 0, math.sin(b)], [0, 1, 0], [-math.sin(b), 0, math.cos(b)]])
    rx = np.array([[1, 0, 0], [0, math.cos(c), -math.sin(c)], [0, math.sin(c), math.cos(c)]])
    return rz @ ry @ rx


class Rng:
    """splitmix64 stream (seeded, platform independent)."""

    def __init__(self, seed):
        self.s = seed & 0xFFFFFFFFFFFFFFFF

    def u64(self):
        self.s = (self.s + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
        z = self.s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
        return z ^ (z >> 31)

    def uniform(self, lo=0.0, hi=1.0):
        return lo + (hi - lo) * ((self.u64() >> 11) * (1.0 / (1 << 53)))

    def vec(self, lo, hi, n=3):
        return np.array([self.uniform(lo, hi) for _ in range(n)])


class Scene:
    """Analytic primitives: rectangles, spheres, axis-aligned boxes."""

    def __init__(self, seed):
        self.seed = seed
        self.rects = []    # (center, axis_u (half extent), axis_v (half extent), normal)
        self.spheres = []  # (center, radius)
        self.boxes = []    # (lo, hi, inward)
        self.patches = []  # (center, radius, (Y, U, V))

    def add_rect(self, center, normal, half_u, half_v, rng):
        n = np.asarray(normal, float)
        n = n / np.linalg.norm(n)
        a = np.cross(n, [0.0, 0.0, 1.0])
        if np.linalg.norm(a) < 1e-6:
            a = np.cross(n, [0.0, 1.0, 0.0])
        a = a / np.linalg.norm(a)
        b = np.cross(n, a)
        ang = rng.uniform(0, math.pi)
        u = math.cos(ang) * a + math.sin(ang) * b
        v = np.cross(n, u)
        self.rects.append((np.asarray(center, float), u * half_u, v * half_v, n))


_sg = None


def _scenegen():
    """ctypes handle of libscenegen.so (the C++ ray caster, built by build.py)."""
    global _sg
    if _sg is None:
        import ctypes
        path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "lib",
                            "libscenegen.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing (run rvs-cuda_b200/build.py)")
        L = ctypes.CDLL(path)
        P = ctypes.c_void_p
        L.sg_render.argtypes = [P, P, P, ctypes.c_int, P, ctypes.c_int, P, ctypes.c_int, P, ctypes.c_int,
                                ctypes.c_uint64, P, P, P, P]
        _sg = L
    return _sg


def render(scene, cam):
    """Renders (Y, U, V, depth) uint16 planes of camera `cam`: per pixel the
    closest hit along the camera ray (perspective: x component 1, so hit
    distance = stored depth; ERP: unit rays, hit distance = radius), misses
    at the far plane, value-noise texture, 2x2-averaged chroma and the
    normalised-disparity depth encoding."""
    w, h = cam.width, cam.height
    ci = np.array([cam.projection, w, h, cam.bit_depth_color, cam.bit_depth_depth], np.int32)
    R = rotation_matrix(cam.rotation)
    cd = np.array(list(cam.position) + list(R.ravel()) + list(cam.focal) + list(cam.principle_point) +
                  list(cam.hor_range) + list(cam.ver_range) + [cam.depth_range[0], cam.depth_range[1]],
                  np.float64)
    rects = np.array([np.concatenate([c, au, av, n]) for c, au, av, n in scene.rects],
                     np.float64).reshape(-1, 12)
    sph = np.array([np.concatenate([c, [r]]) for c, r in scene.spheres], np.float64).reshape(-1, 4)
    boxes = np.array([np.concatenate([lo, hi, [1.0 if inward else 0.0]]) for lo, hi, inward in scene.boxes],
                     np.float64).reshape(-1, 7)
    pat = np.array([np.concatenate([c, [r], col]) for c, r, col in scene.patches], np.float64).reshape(-1, 7)
    Y = np.empty((h, w), np.uint16)
    U = np.empty((h // 2, w // 2), np.uint16)
    V = np.empty((h // 2, w // 2), np.uint16)
    D = np.empty((h, w), np.uint16)
    rc = _scenegen().sg_render(ci.ctypes.data, cd.ctypes.data, rects.ctypes.data, len(rects), sph.ctypes.data,
                               len(sph), boxes.ctypes.data, len(boxes), pat.ctypes.data, len(pat),
                               scene.seed & 0xFFFFFFFFFFFFFFFF, Y.ctypes.data, U.ctypes.data, V.ctypes.data,
                               D.ctypes.data)
    if rc != 0:
        raise ValueError("scene render failed (odd or empty resolution)")
    return Y, U, V, D


def _front_scene(seed, n_planes, n_spheres, dmin, dmax, spread):
    rng = Rng(seed)
    sc = Scene(seed)
    for _ in range(n_planes):
        x = rng.uniform(dmin, dmax)
        c = np.array([x, rng.uniform(-spread, spread) * x, rng.uniform(-spread * 0.6, spread * 0.6) * x])
        nrm = np.array([-1.0, rng.uniform(-0.6, 0.6), rng.uniform(-0.5, 0.5)])
        sc.add_rect(c, nrm, rng.uniform(0.4, 0.5 * x), rng.uniform(0.3, 0.4 * x), rng)
    for _ in range(n_spheres):
        x = rng.uniform(dmin, dmax)
        c = np.array([x, rng.uniform(-spread, spread) * x, rng.uniform(-spread * 0.5, spread * 0.5) * x])
        sc.spheres.append((c, rng.uniform(0.15, 0.12 * x + 0.2)))
    # Flat-colour patches centred near the primitives.
    prims = [r[0] for r in sc.rects] + [s[0] for s in sc.spheres]
    for k in range(8):
        c = prims[k % len(prims)] + rng.vec(-0.3, 0.3)
        sc.patches.append((c, rng.uniform(0.2, 0.5),
                           (rng.uniform(0.1, 0.9), rng.uniform(0.3, 0.7), rng.uniform(0.3, 0.7))))
    return sc


class Workload:
    """Input cameras + rendered planes + target cameras."""

    def __init__(self, name, scene, inputs, targets, blending_factor=5.0):
        self.name = name
        self.scene = scene
        self.inputs = inputs
        self.targets = targets
        self.blending_factor = blending_factor
        self._planes = None

    @property
    def planes(self):
        if self._planes is None:
            self._planes = [render(self.scene, c) for c in self.inputs]
        return self._planes


def plain_small(scale=1.0, seed=0x5EED0001):
    """2 perspective inputs 960x540 (f = 800, principal point at the centre)
    0.1 m apart on a horizontal line; 1 target at the midpoint.  `scale`
    shrinks the images (and the focal length) for CPU-sized tests."""
    w, h = _even(960 * scale), _even(540 * scale)
    f = 800.0 * w / 960.0
    sc = _front_scene(seed, 3, 2, 1.2, 8.0, 0.35)
    mk = lambda y: abi.make_camera(abi.PERSPECTIVE, w, h, (0, y, 0), (0, 0, 0), (0.5, 10.0), (f, f))
    inputs = [mk(0.05), mk(-0.05)]
    targets = [mk(0.0)]
    return Workload("plain_small", sc, inputs, targets)


def plain_1080p(scale=1.0, seed=0x5EED0002, n_targets=1):
    """4 perspective inputs 1920x1080 (f = 1500) on a 2x2 grid, 0.15 m
    spacing; targets at seeded poses inside the grid (+-7.5 cm in y and z,
    +-10 cm in x, +-5 degrees); the first is the plain workload's view."""
    w, h = _even(1920 * scale), _even(1080 * scale)
    f = 1500.0 * w / 1920.0
    sc = _front_scene(seed, 6, 4, 1.0, 8.0, 0.3)
    rng = Rng(seed ^ 0xABCDEF)
    inputs = [abi.make_camera(abi.PERSPECTIVE, w, h, (0, y, z), (0, 0, 0), (0.5, 10.0), (f, f))
              for z in (0.075, -0.075) for y in (0.075, -0.075)]
    targets = []
    for _ in range(n_targets):
        pos = (rng.uniform(-0.1, 0.1), rng.uniform(-0.075, 0.075), rng.uniform(-0.075, 0.075))
        rot = (rng.uniform(-5, 5), rng.uniform(-5, 5), rng.uniform(-5, 5))
        targets.append(abi.make_camera(abi.PERSPECTIVE, w, h, pos, rot, (0.5, 10.0), (f, f)))
    return Workload("plain_1080p", sc, inputs, targets)


def _room_scene(seed):
    rng = Rng(seed)
    sc = Scene(seed)
    lo, hi = np.array([-4.0, -3.0, -1.5]), np.array([4.0, 3.0, 1.5])
    sc.boxes.append((lo, hi, True))
    for k in range(12):
        c = np.array([rng.uniform(-3, 3), rng.uniform(-2.2, 2.2), rng.uniform(-1.0, 1.0)])
        if np.linalg.norm(c) < 1.2:
            c = c / np.linalg.norm(c) * 1.2
        if k % 2 == 0:
            sc.spheres.append((c, rng.uniform(0.2, 0.5)))
        else:
            e = rng.uniform(0.15, 0.4)
            sc.boxes.append((c - e, c + e, False))
    for k in range(8):
        c = np.array([rng.uniform(-4, 4), rng.uniform(-3, 3), rng.uniform(-1.5, 1.5)])
        sc.patches.append((c, rng.uniform(0.3, 0.8),
                           (rng.uniform(0.1, 0.9), rng.uniform(0.3, 0.7), rng.uniform(0.3, 0.7))))
    return sc


def catmull_rom(points, n):
    """n samples along a closed Catmull-Rom spline through points (K, 3)."""
    k = len(points)
    out = []
    for i in range(n):
        t = i * k / n
        s = int(t)
        u = t - s
        p0, p1, p2, p3 = (points[(s + d) % k] for d in (-1, 0, 1, 2))
        out.append(0.5 * ((2 * p1) + (-p0 + p2) * u + (2 * p0 - 5 * p1 + 4 * p2 - p3) * u * u +
                          (-p0 + 3 * p1 - 3 * p2 + p3) * u ** 3))
    return out


def batched_erp(scale=1.0, n_targets=300, seed=0x5EED0003):
    """4 ERP 360x180 inputs 4096x2048 (near 0.3 m, far 20 m) at the vertices
    of a tetrahedron 0.2 m from the centre of a room-box scene; perspective
    1920x1080 targets with 90 degrees horizontal field of view along a seeded
    closed Catmull-Rom trajectory."""
    w, h = _even(4096 * scale), _even(2048 * scale)
    sc = _room_scene(seed)
    rng = Rng(seed ^ 0x777)
    s = 0.2 / math.sqrt(3)
    verts = [(s, s, s), (s, -s, -s), (-s, s, -s), (-s, -s, s)]
    inputs = [abi.make_camera(abi.EQUIRECTANGULAR, w, h, v, (0, 0, 0), (0.3, 20.0),
                              hor_range=(-180, 180), ver_range=(-90, 90)) for v in verts]
    wo, ho = _even(1920 * scale), _even(1080 * scale)
    f = wo / 2.0  # 90 degrees horizontal field of view
    ctrl = [np.array([rng.uniform(-0.1, 0.1), rng.uniform(-0.1, 0.1), rng.uniform(-0.05, 0.05)])
            for _ in range(8)]
    yaw0 = rng.uniform(-180, 180)
    pos = catmull_rom(ctrl, n_targets)
    targets = []
    for i, p in enumerate(pos):
        rot = (yaw0 + 360.0 * i / max(n_targets, 1), 8.0 * math.sin(i * 0.05), 3.0 * math.sin(i * 0.03))
        targets.append(abi.make_camera(abi.PERSPECTIVE, wo, ho, p, rot, (0.3, 20.0), (f, f)))
    return Workload("batched_erp", sc, inputs, targets)


def batched_mixed(scale=1.0, n_targets=64, seed=0x5EED0004):
    """11 perspective inputs 2048x1088 on a 3x4 grid (one missing), 0.1 m
    spacing, in front of 20 planes and 10 spheres; targets mix 960x540,
    1920x1080 and 2048x1088."""
    w, h = _even(2048 * scale), _even(1088 * scale)
    f = 1600.0 * w / 2048.0
    sc = _front_scene(seed, 20, 10, 1.0, 9.0, 0.35)
    rng = Rng(seed ^ 0x999)
    inputs = []
    for r in range(3):
        for c in range(4):
            if (r, c) == (1, 3):
                continue
            inputs.append(abi.make_camera(abi.PERSPECTIVE, w, h, (0, 0.15 - 0.1 * c, 0.1 - 0.1 * r),
                                          (0, 0, 0), (0.5, 12.0), (f, f)))
    sizes = [(960, 540), (1920, 1080), (2048, 1088)]
    targets = []
    for i in range(n_targets):
        tw, th = sizes[i % 3]
        tw, th = _even(tw * scale), _even(th * scale)
        tf = f * tw / w
        pos = (rng.uniform(-0.05, 0.05), rng.uniform(-0.15, 0.15), rng.uniform(-0.1, 0.1))
        rot = (rng.uniform(-4, 4), rng.uniform(-4, 4), rng.uniform(-2, 2))
        targets.append(abi.make_camera(abi.PERSPECTIVE, tw, th, pos, rot, (0.5, 12.0), (tf, tf)))
    return Workload("batched_mixed", sc, inputs, targets)


def _even(x):
    x = int(round(x))
    return max(2, x - (x & 1))


def random_pose_small(n_views=2, w=64, h=36, seed=1, erp_out=False, erp_in=False):
    """Small random workloads for parity tests (a few seconds on the CPU)."""
    rng = Rng(seed)
    sc = _front_scene(seed, 3, 2, 1.0, 6.0, 0.35) if not erp_in else _room_scene(seed)
    f = 0.8 * w
    inputs = []
    for k in range(n_views):
        pos = (rng.uniform(-0.05, 0.05), rng.uniform(-0.1, 0.1), rng.uniform(-0.06, 0.06))
        if erp_in:
            inputs.append(abi.make_camera(abi.EQUIRECTANGULAR, w, h, pos, (0, 0, 0), (0.3, 20.0)))
        else:
            rot = (rng.uniform(-3, 3), rng.uniform(-3, 3), rng.uniform(-2, 2))
            inputs.append(abi.make_camera(abi.PERSPECTIVE, w, h, pos, rot, (0.5, 10.0), (f, f)))
    pos = (rng.uniform(-0.05, 0.05), rng.uniform(-0.08, 0.08), rng.uniform(-0.05, 0.05))
    if erp_out:
        tgt = abi.make_camera(abi.EQUIRECTANGULAR, w, h, pos, (rng.uniform(-20, 20), 0, 0),
                              (0.3, 20.0))
    else:
        rot = (rng.uniform(-4, 4), rng.uniform(-4, 4), rng.uniform(-3, 3))
        near_far = (0.3, 20.0) if erp_in else (0.5, 10.0)
        tgt = abi.make_camera(abi.PERSPECTIVE, w, h, pos, rot, near_far, (f, f))
    return Workload("random_small", sc, inputs, [tgt])


WORKLOADS = {
    "plain_small": plain_small,
    "plain_1080p": plain_1080p,
    "batched_erp": batched_erp,
    "batched_mixed": batched_mixed,
}


def cache_planes(workload, cache_dir):
    """Renders (or loads from cache_dir) the input planes of a workload."""
    os.makedirs(cache_dir, exist_ok=True)
    key = f"{workload.name}_{workload.inputs[0].width}x{workload.inputs[0].height}_{workload.scene.seed:x}.npz"
    path = os.path.join(cache_dir, key)
    if os.path.exists(path):
        z = np.load(path)
        workload._planes = [(z[f"y{i}"], z[f"u{i}"], z[f"v{i}"], z[f"d{i}"])
                            for i in range(len(workload.inputs))]
        return workload.planes
    planes = workload.planes
    np.savez(path, **{f"{k}{i}": p[j] for i, p in enumerate(planes)
                      for j, k in enumerate("yuvd")})
    return planes
