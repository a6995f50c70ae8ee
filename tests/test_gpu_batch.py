"""Batched rendering (vpt_batch_*): several independent scenes traced by one persistent launch, with
and without the captured CUDA graph, must give every scene exactly the film it gets when rendered
alone (same paths; FP64 film equal up to the order of the atomic additions) in the parity build."""
import ctypes

import numpy as np
import pytest

from cloudrendering_b200._lib import VptStats
from oracle import bridge
from tests.harness import Core, SceneSpec, cloud_block, setup_core

pytestmark = pytest.mark.gpu

FRAMES = [1, 3, 2, 4]


def scenes(mode):
    base = dict(albedo=0.99, env="constant_sun", sky_color=(0.2, 0.2, 0.2), sun_intensity=(5.0, 5.0, 5.0),
                linear_rgb=1, max_grid_extent=0.5, max_bounces=64, mode=mode)
    return [
        SceneSpec(grid=bridge.fbm(24, 2, base_frequency=3.0, contrast=3.5), extinction=120.0, g=0.85, width=32,
                  height=32, cam_pos=(0.3, 0.4, 1.4), sun_dir=(0.3, 0.8, 0.5), **base),
        SceneSpec(grid=bridge.fbm((40, 24, 33), 7, base_frequency=3.0, contrast=3.5), extinction=300.0, g=0.6,
                  width=48, height=40, cam_pos=(-1.2, 0.3, 0.9), sun_dir=(-0.2, 0.9, 0.1), seed_offset=17, **base),
        SceneSpec(grid=cloud_block(8, 8, 8, empty_boundary=True), extinction=60.0, g=0.7, width=64, height=24,
                  cam_pos=(0.0, 0.2, 1.6), sun_dir=(0.5, 0.5, 0.5), **base),
        SceneSpec(grid=bridge.fbm(40, 3, base_frequency=2.0, contrast=12.0), extinction=500.0, g=0.9, width=20,
                  height=36, cam_pos=(1.0, 1.0, 1.0), sun_dir=(0.0, 1.0, 0.2), **base),
    ]


def films(cores, sps):
    out = []
    for c, sp in zip(cores, sps):
        s = np.zeros(sp.width * sp.height * 3, np.float64)
        c("vpt_read_statistics", s.ctypes.data_as(ctypes.c_void_p), None, 0, None)
        out.append(s)
    return out


@pytest.fixture(scope="module", params=["dr", "default"])
def cores(request):
    """The parity build (no FMA contraction anywhere) and the product build, whose batch and
    single-scene kernels sit in different units and may contract multiply-adds differently."""
    cs = [Core(0, request.param) for _ in range(4)]
    for c in cs:
        c.variant = request.param
    yield cs
    for c in cs:
        c.close()


def make_batch(cores):
    lib = cores[0].lib
    arr = (ctypes.c_void_p * len(cores))(*[c.ctx for c in cores])
    b = ctypes.c_void_p()
    assert lib.vpt_batch_create(ctypes.byref(b), arr, len(cores)) == 0
    return b


def check(lib, b, st):
    assert st == 0, lib.vpt_batch_last_error(b)


@pytest.mark.parametrize("mode", ["delta", "ratio", "nee"])
@pytest.mark.parametrize("use_graph", [1, 0])
def test_batch_equals_individual_renders(cores, mode, use_graph):
    sps = scenes(mode)
    lib = cores[0].lib
    for c, sp in zip(cores, sps):
        setup_core(c, sp)
        c("vpt_set_collect_statistics", 0)
    # alone: two calls per scene
    for c, f in zip(cores, FRAMES):
        c("vpt_reset_accumulation")
        c("vpt_render_frames", f, None)
        c("vpt_render_frames", f, None)
        c("vpt_synchronize", None)
    alone = films(cores, sps)
    # batched: two calls (with the graph, the second one replays the captured launch)
    b = make_batch(cores)
    try:
        check(lib, b, lib.vpt_batch_set_option(b, b"use_graph", float(use_graph)))
        for c in cores:
            c("vpt_reset_accumulation")
        frames = (ctypes.c_int * 4)(*FRAMES)
        check(lib, b, lib.vpt_batch_render(b, frames, None))
        check(lib, b, lib.vpt_batch_render(b, frames, None))
        for c in cores:
            c("vpt_synchronize", None)
        batched = films(cores, sps)
        for a, bb in zip(alone, batched):
            assert np.all(np.isfinite(bb))
            if cores[0].variant == "dr":
                assert np.allclose(a, bb, rtol=1e-12, atol=1e-12)
            else:
                # a last-ulp difference of a contracted multiply-add can send a path another way, so
                # the product build's films agree in the image sum and in most pixels
                assert abs(a.sum() - bb.sum()) <= 0.02 * abs(a.sum())
                assert np.mean(np.isclose(a, bb, rtol=1e-3, atol=1e-6)) >= 0.5
    finally:
        lib.vpt_batch_destroy(b)


def test_batch_autotune_and_stats(cores):
    sps = scenes("delta")
    lib = cores[0].lib
    for c, sp in zip(cores, sps):
        setup_core(c, sp)
    b = make_batch(cores)
    try:
        frames = (ctypes.c_int * 4)(*FRAMES)
        best = ctypes.c_int()
        check(lib, b, lib.vpt_batch_autotune(b, frames, None, ctypes.byref(best)))
        assert 1 <= best.value <= 64
        check(lib, b, lib.vpt_batch_reset_stats(b))
        check(lib, b, lib.vpt_batch_render(b, frames, None))
        st = VptStats()
        check(lib, b, lib.vpt_batch_get_stats(b, ctypes.byref(st)))
        assert st.paths == sum(sp.width * sp.height * f for sp, f in zip(sps, FRAMES))
        assert st.density_lookups > 0 and st.error_flags == 0
    finally:
        lib.vpt_batch_destroy(b)


def test_batch_rejects_mixed_trackers(cores):
    sps = scenes("delta")
    sps[1].mode = "nee"
    for c, sp in zip(cores, sps):
        setup_core(c, sp)
    lib = cores[0].lib
    b = make_batch(cores)
    try:
        frames = (ctypes.c_int * 4)(*FRAMES)
        assert lib.vpt_batch_render(b, frames, None) == 6  # VPT_ERR_UNSUPPORTED
    finally:
        lib.vpt_batch_destroy(b)
