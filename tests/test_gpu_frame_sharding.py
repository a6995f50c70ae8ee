"""Frame sharding on the CUDA core (vpt_set_frame_index): contexts that render disjoint frame ranges
of one image trace exactly the paths of one context rendering all frames, so their FP64 films sum to
its film (equal up to the order of the atomic additions).  The frame origin survives parameter
changes, which clear the film back to it."""
import ctypes

import numpy as np
import pytest

from oracle import bridge
from tests.harness import Core, SceneSpec, setup_core

pytestmark = pytest.mark.gpu

TOTAL = 10
SPLITS = [(0, 3), (3, 4), (7, 3)]


def film(c, sp):
    s = np.zeros(sp.width * sp.height * 3, np.float64)
    c("vpt_read_statistics", s.ctypes.data_as(ctypes.c_void_p), None, 0, None)
    return s


@pytest.fixture(scope="module")
def cores():
    cs = [Core(0) for _ in range(len(SPLITS) + 1)]
    yield cs
    for c in cs:
        c.close()


@pytest.mark.parametrize("mode", ["delta", "nee"])
def test_disjoint_frame_ranges_sum_to_one_render(cores, mode):
    sp = SceneSpec(grid=bridge.fbm(32, 5, base_frequency=3.0, contrast=3.5), extinction=200.0, albedo=0.99, g=0.85,
                   width=40, height=32, env="constant_sun", sky_color=(0.2, 0.2, 0.2), sun_intensity=(5.0, 5.0, 5.0),
                   sun_dir=(0.3, 0.8, 0.5), cam_pos=(0.3, 0.4, 1.4), linear_rgb=1, max_grid_extent=0.5,
                   max_bounces=64, mode=mode)
    whole, parts = cores[0], cores[1:]
    setup_core(whole, sp)
    whole("vpt_set_frame_index", 0)
    whole("vpt_render_frames", TOTAL, None)
    whole("vpt_synchronize", None)
    ref = film(whole, sp)
    acc = np.zeros_like(ref)
    for c, (first, n) in zip(parts, SPLITS):
        c("vpt_set_frame_index", first)
        setup_core(c, sp)  # parameter changes clear the film back to the frame origin
        c("vpt_render_frames", n, None)
        c("vpt_synchronize", None)
        acc += film(c, sp)
        c("vpt_set_frame_index", 0)
    assert np.all(np.isfinite(acc)) and ref.sum() > 0
    assert np.allclose(acc, ref, rtol=1e-11, atol=1e-12)
