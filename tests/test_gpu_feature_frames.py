"""The feature frame limit (vpt_set_option "feature_frames"): feature maps accumulate over the first k
frames only and later frames are traced without the feature pass.  The film is the same as without
the limit (the feature pass draws no random numbers, so every path is the same), and the feature
maps equal those of a render of only the first k frames."""
import ctypes

import numpy as np
import pytest

from oracle import bridge
from tests.harness import Core, SceneSpec, setup_core

pytestmark = pytest.mark.gpu

FEATURES = {"albedo": 17, "normal": 3, "depth": 6}


def film(c, sp):
    s = np.zeros(sp.width * sp.height * 3, np.float64)
    c("vpt_read_statistics", s.ctypes.data_as(ctypes.c_void_p), None, 0, None)
    return s


def feature(c, sp, fid, ch=2):
    out = np.zeros(ch * sp.width * sp.height, np.float32)
    c("vpt_get_feature_map", fid, out.ctypes.data_as(ctypes.c_void_p), ch, 0, None)
    return out


@pytest.mark.parametrize("mode", ["delta", "nee"])
def test_feature_frame_limit(mode):
    sp = SceneSpec(grid=bridge.fbm(32, 5, base_frequency=3.0, contrast=3.5), extinction=200.0, albedo=0.99, g=0.85,
                   width=48, height=40, env="constant_sun", sky_color=(0.2, 0.2, 0.2), sun_intensity=(5.0, 5.0, 5.0),
                   sun_dir=(0.3, 0.8, 0.5), cam_pos=(0.3, 0.4, 1.4), linear_rgb=1, max_grid_extent=0.5,
                   max_bounces=64, mode=mode)
    ids = (ctypes.c_int * 3)(*FEATURES.values())
    # the parity build: the limited render mixes the feature kernel and the refill kernel, whose
    # operations the product build may contract into FMAs differently
    cores = [Core(0, "dr") for _ in range(3)]
    try:
        limited, full, short = cores
        for c in cores:
            setup_core(c, sp)
            c("vpt_set_use_feature_maps", ids, 3)
        limited("vpt_set_option", b"feature_frames", 2.0)
        limited("vpt_render_frames", 3, None)
        limited("vpt_render_frames", 3, None)
        full("vpt_render_frames", 6, None)
        short("vpt_render_frames", 2, None)
        for c in cores:
            c("vpt_synchronize", None)
        assert np.allclose(film(limited, sp), film(full, sp), rtol=1e-11, atol=1e-12)
        for fid in FEATURES.values():
            a, b = feature(limited, sp, fid), feature(short, sp, fid)
            assert np.allclose(a, b, rtol=1e-5, atol=1e-6), fid
            assert not np.allclose(a, feature(full, sp, fid), rtol=1e-3, atol=1e-4) or fid == 17
    finally:
        for c in cores:
            c.close()
