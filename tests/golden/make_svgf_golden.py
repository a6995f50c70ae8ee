"""Generates tests/golden/svgf_frames.npz from the reference's own SVGF compute shaders run on the CPU
(Data/Shaders/Denoiser/SVGF/SVGF.glsl: reprojection, moments filter, a-trous; oracle/_ref/libref_image.so
built by oracle/ref_build.py, the pass sequence of SVGFDenoiser::denoise in ref_image_driver.cpp).

Five frames of synthetic maps (smooth depth with a step edge, normals with a crease, noisy colour, zero
then sub-pixel motion; tests/test_gpu_svgf.py's generator) for 5, 1 and 0 a-trous iterations: the
inputs, then per frame the filtered image and the colour / moments history after the frame.

Run in a container that has the reference tree:  python tests/golden/make_svgf_golden.py
"""
import ctypes
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import ref_build  # noqa: E402
from tests.test_gpu_svgf import maps  # noqa: E402

H, W, FRAMES = 32, 40, 5
Z_THRESHOLD, NORMAL_THRESHOLD = 0.2, 0.2


def main():
    ref_build.build()
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_image.so"))
    P = ctypes.c_void_p
    data = {}
    g = np.random.default_rng(7)
    inputs = [maps(H, W, f, g) for f in range(FRAMES)]
    for f, arrs in enumerate(inputs):
        for name, a in zip(("noisy", "normal", "depth", "fwidth", "motion"), arrs):
            data[f"in{f}__{name}"] = a
    for iterations in (5, 1, 0):
        hist = {"color": np.zeros((H, W, 4), np.float32), "moments": np.zeros((H, W, 4), np.float32),
                "normal": np.zeros((H, W, 4), np.float32), "depth": np.zeros((H, W), np.float32)}
        for f, arrs in enumerate(inputs):
            out = np.zeros((H, W, 4), np.float32)
            assert lib.ref_svgf_frame(*[a.ctypes.data_as(P) for a in arrs],
                                      *[hist[k].ctypes.data_as(P) for k in ("color", "moments", "normal", "depth")],
                                      W, H, ctypes.c_float(Z_THRESHOLD), ctypes.c_float(NORMAL_THRESHOLD), iterations,
                                      out.ctypes.data_as(P)) == 0
            data[f"it{iterations}_f{f}__out"] = out
            data[f"it{iterations}_f{f}__color"] = hist["color"].copy()
            data[f"it{iterations}_f{f}__moments"] = hist["moments"].copy()
            print(iterations, f, float(out[..., :3].mean()), float(hist["moments"][..., 2].max()))
    meta = {"h": H, "w": W, "frames": FRAMES, "iterations": [5, 1, 0], "z_threshold": Z_THRESHOLD,
            "normal_threshold": NORMAL_THRESHOLD}
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "svgf_frames.npz")
    np.savez_compressed(path, meta=json.dumps(meta), **data)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
