"""Generates the golden fixtures under tests/golden/.

1. cv2_resize_half.npz: the OpenCV behaviour the writer depends on
   (write_color_YUV, rvs/src/image_writing.cpp:83-84: cv::resize(0.5, 0.5,
   INTER_LINEAR) of quantised uint16 chroma planes), recorded from the
   Python cv2 wheel available in the build container.
2. cv2_norm_vec2f.npz: cv::norm of two cv::Vec2f (valid_tri,
   rvs/src/transform.cpp:63-65), recorded from cv2.norm on float32 pairs.
3. synth_small_*.npz: small seeded syntheses by the CPU oracle (inputs,
   cameras, blended quality and the YUV420 result), which pin the oracle
   against later changes and give the GPU tests fixed expected outputs.
4. cv2_resize_nearest.npz: cv::resize with INTER_NEAREST of one-byte masks
   from the raster sizes of Precision != 1 to the output size (the validity
   mask, Pipeline.cpp:303-308), recorded from cv2.

Run from the repository root: python tests/golden/make_golden.py [NAME...]
(NAME: resize_half, norm, synth, resize_nearest; all by default; needs
cv2; the tests themselves only read the .npz files).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "rvs-cuda_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def camera_to_array(c):
    from rvsb import abi
    raw = bytes(c)
    return np.frombuffer(raw, np.uint8).copy()


def resize_nearest():
    import cv2
    rng = np.random.default_rng(20261204)
    arrays = {}
    # (output w, h) and Precision: the raster is int(0.5 + W * P) x int(0.5 + H * P)
    cases = [(128, 64, 2.0), (128, 64, 1.5), (96, 54, 1.5), (128, 64, 0.75), (100, 50, 0.9), (64, 36, 0.5),
             (1920, 1080, 1.5), (960, 540, 0.7)]
    for k, (w, h, P) in enumerate(cases):
        P32 = np.float32(P)
        rw, rh = int(np.float32(0.5) + np.float32(w) * P32), int(np.float32(0.5) + np.float32(h) * P32)
        m = (rng.random((rh, rw)) < 0.3).astype(np.uint8) * 255
        arrays[f"in{k}"] = m
        arrays[f"out{k}"] = cv2.resize(m, (w, h), interpolation=cv2.INTER_NEAREST)
    np.savez_compressed(os.path.join(HERE, "cv2_resize_nearest.npz"), n=len(cases), **arrays)


def main(names=("resize_half", "norm", "synth", "resize_nearest")):
    import cv2
    import oracle as O
    from rvsb import scenes

    if "resize_nearest" in names:
        resize_nearest()
    if not {"resize_half", "norm", "synth"} & set(names):
        print("golden fixtures written to", HERE)
        return
    rng = np.random.default_rng(20261203)
    # 1. cv::resize(0.5, 0.5, INTER_LINEAR) of uint16 planes
    #    recorded with Intel IPP on (outK, ties to even) and off (outK_noipp,
    #    ties up): the result depends on how OpenCV was built.
    shapes = [(2, 2), (4, 6), (16, 32), (64, 96), (36, 64)]
    arrays = {}

    def resize_both(a):
        out = []
        for ipp in (True, False):
            cv2.ipp.setUseIPP(ipp)
            out.append(cv2.resize(a, None, fx=0.5, fy=0.5, interpolation=cv2.INTER_LINEAR))
        cv2.ipp.setUseIPP(True)
        return out

    for k, (h, w) in enumerate(shapes):
        a = rng.integers(0, 1024, size=(h, w), dtype=np.uint16)
        if k == 0:
            a = np.array([[0, 1], [3, 3]], np.uint16)
        arrays[f"in{k}"] = a
        arrays[f"out{k}"], arrays[f"out{k}_noipp"] = resize_both(a)
    arrays["full_range_in"] = rng.integers(0, 65536, size=(32, 32), dtype=np.uint16)
    arrays["full_range_out"], arrays["full_range_out_noipp"] = resize_both(arrays["full_range_in"])
    arrays["ipp_available"] = np.int32(cv2.ipp.useIPP())
    np.savez_compressed(os.path.join(HERE, "cv2_resize_half.npz"), n=len(shapes), **arrays)

    # 2. cv::norm(Vec2f, Vec2f)
    n = 4000
    a = (rng.standard_normal((n, 2)) * rng.choice([1e-3, 1.0, 40.0, 3000.0], size=(n, 1))).astype(np.float32)
    b = (a + rng.standard_normal((n, 2)).astype(np.float32) * rng.choice([1e-4, 0.5, 2.0, 100.0], size=(n, 1))
         ).astype(np.float32)
    norms = np.array([cv2.norm(a[k], b[k]) for k in range(n)], np.float64)
    np.savez_compressed(os.path.join(HERE, "cv2_norm_vec2f.npz"), a=a, b=b, norm=norms)

    # 3. oracle regression cases
    cases = [dict(n_views=2, w=64, h=36, seed=101), dict(n_views=3, w=96, h=54, seed=102),
             dict(n_views=2, w=128, h=64, seed=103, erp_in=True, erp_out=True)]
    for k, case in enumerate(cases):
        wl = scenes.random_pose_small(**case)
        target = wl.targets[0]
        (Y, U, V), q, c = O.synthesize(wl.inputs, wl.planes, target, 5.0, want_intermediate=True)
        data = {"Y": Y, "U": U, "V": V, "quality": q, "exponent": np.float32(5.0),
                "target": camera_to_array(target), "n": len(wl.inputs)}
        for i, (cam, (y, u, v, d)) in enumerate(zip(wl.inputs, wl.planes)):
            data[f"cam{i}"] = camera_to_array(cam)
            data[f"y{i}"], data[f"u{i}"], data[f"v{i}"], data[f"d{i}"] = y, u, v, d
        np.savez_compressed(os.path.join(HERE, f"synth_small_{k}.npz"), **data)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main(tuple(sys.argv[1:]) or ("resize_half", "norm", "synth", "resize_nearest"))
