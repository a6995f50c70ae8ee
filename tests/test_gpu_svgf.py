"""SVGF (Data/Shaders/Denoiser/SVGF/SVGF.glsl) on the CUDA core against the CPU oracle's restatement
(oracle_svgf_frame): several frames of synthetic maps (smooth depth with a step edge, normals with
a crease, noisy colour, zero and sub-pixel motion), the filtered image and every history buffer,
through vpt_svgf_filter.  Both sides compute in float without FMA contraction; expf/powf differ in
the last ulp, so values agree to rtol 1e-4 (a validity test or bilinear branch that flips on such a
difference is allowed for 0.1 % of the pixels)."""
import ctypes

import numpy as np
import pytest
import torch

from cloudrendering_b200 import _lib
from oracle import bridge

pytestmark = pytest.mark.gpu


def maps(h, w, frame, g):
    ys, xs = np.mgrid[0:h, 0:w].astype(np.float32)
    depth = (1.5 + 0.002 * xs + 0.001 * ys + np.where(xs > w * 0.6, 0.3, 0.0)).astype(np.float32)
    nrm = np.zeros((h, w, 4), np.float32)
    nrm[..., 2] = 1.0
    nrm[ys > h / 2, 0] = 0.6
    nrm[ys > h / 2, 2] = 0.8
    base = 0.5 + 0.4 * np.sin(xs / 7.0)[..., None] * np.array([1.0, 0.8, 0.6], np.float32)
    noisy = np.concatenate([base + g.exponential(0.3, (h, w, 3)) - 0.3, np.ones((h, w, 1))], -1).astype(np.float32)
    fw = np.full((h, w), 0.003, np.float32)
    motion = np.zeros((h, w, 2), np.float32)
    if frame >= 2:
        motion[..., 0], motion[..., 1] = 1.3, -0.6
    return noisy, nrm, depth, fw, motion


@pytest.mark.parametrize("iterations", [5, 1, 0])
def test_svgf_frames_match_the_oracle(iterations):
    lib = _lib.load()
    torch.cuda.init()
    h, w = 48, 64
    g = np.random.default_rng(7)
    hist_o = {"color": np.zeros((h, w, 4), np.float32), "moments": np.zeros((h, w, 4), np.float32),
              "normal": np.zeros((h, w, 4), np.float32), "depth": np.zeros((h, w), np.float32)}
    hist_g = {k: torch.zeros(v.shape, dtype=torch.float32, device="cuda") for k, v in hist_o.items()}
    for frame in range(5):
        noisy, nrm, depth, fw, motion = maps(h, w, frame, g)
        ref = bridge.svgf_frame(noisy, nrm, depth, fw, motion, hist_o, 0.002 * 100, 0.02 * 10, iterations)
        dev = [torch.from_numpy(a).cuda() for a in (noisy, nrm, depth, fw, motion)]
        out = torch.empty((h, w, 4), dtype=torch.float32, device="cuda")
        p = lambda t: ctypes.c_void_p(t.data_ptr())
        st = lib.vpt_svgf_filter(*[p(t) for t in dev], p(hist_g["color"]), p(hist_g["moments"]), p(hist_g["normal"]),
                                 p(hist_g["depth"]), w, h, ctypes.c_float(0.2), ctypes.c_float(0.2), iterations, p(out),
                                 None)
        assert st == 0
        torch.cuda.synchronize()
        for name, got, exp in [("out", out.cpu().numpy(), ref)] + [(k, hist_g[k].cpu().numpy(), hist_o[k])
                                                                  for k in hist_o]:
            assert np.all(np.isfinite(got)), name
            close = np.abs(got - exp) <= 1e-4 * (np.abs(exp) + 1e-3)
            pix = close.reshape(h * w, -1).all(axis=1)
            assert pix.mean() >= 0.999, (frame, name, pix.mean())
            assert np.abs(got - exp).max() <= 0.05 * (np.abs(exp).max() + 1e-3), (frame, name)
        # the history length grows while reprojection succeeds
        assert hist_o["moments"][..., 2].max() == frame + 1


@pytest.mark.parametrize("iterations", [5, 1, 0])
def test_svgf_frames_match_the_reference_shaders(iterations):
    """vpt_svgf_filter against the reference's own SVGF compute shaders run on the CPU
    (tests/golden/svgf_frames.npz), five frames: the image and the colour / moments histories; the same
    tolerance as against the oracle."""
    from tests.harness import svgf_close, svgf_golden

    meta, inputs, outputs = svgf_golden()
    lib = _lib.load()
    h, w = meta["h"], meta["w"]
    hist = {"color": torch.zeros((h, w, 4), device="cuda"), "moments": torch.zeros((h, w, 4), device="cuda"),
            "normal": torch.zeros((h, w, 4), device="cuda"), "depth": torch.zeros((h, w), device="cuda")}
    p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    for f, arrs in enumerate(inputs):
        dev = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in arrs]
        out = torch.empty((h, w, 4), dtype=torch.float32, device="cuda")
        st = lib.vpt_svgf_filter(*[p(t) for t in dev], p(hist["color"]), p(hist["moments"]), p(hist["normal"]),
                                 p(hist["depth"]), w, h, ctypes.c_float(meta["z_threshold"]),
                                 ctypes.c_float(meta["normal_threshold"]), iterations, p(out), None)
        assert st == 0
        torch.cuda.synchronize()
        ref_out, ref_color, ref_moments = outputs[(iterations, f)]
        for name, got, exp in (("out", out, ref_out), ("color", hist["color"], ref_color),
                               ("moments", hist["moments"], ref_moments)):
            assert svgf_close(got.cpu().numpy(), exp) >= 0.999, (f, name)
