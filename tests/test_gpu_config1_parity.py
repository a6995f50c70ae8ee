"""Parity at the reference-sized plain delta-tracking configuration, through the public module API.

Scene: 128^3 fp32 fBm cloud (seed 1, 6 octaves, lacunarity 2, gain 0.5, values below 0.3 set to 0),
unit cube, extinction 200, albedo 0.99, HG g = 0.85, sun 5 from a seeded direction plus constant sky
0.2, 60 degree pinhole camera orbiting at distance 2 (seeded angle), 256x256, 64 spp, at most 64
bounces, fp32 RGBA output; rendered with `vpt.render_frame` on a CUDA tensor.

Checked against the CPU oracle (the restatement of Clouds.glsl / DeltaTracking.glsl, pinned to the
reference shaders compiled for the CPU):
* frame 0: every camera path traced by both from the same seed; >= 99 % agree to rtol 1e-4;
* 64 spp: the GPU image against an oracle render from independent seeds (another seed offset):
  z-test with a Bonferroni bound on 8x8-pixel bins (|z| < 5 over 32*32*3 bins; single pixels are
  heavy-tailed: rare paths see the sun lobe), at most 1 % of pixel-channels beyond |z| = 4, image
  means within |delta| <= 1e-3 per channel (the tolerance of test/TestVolumetricPathTracing.cpp:76-146)
  and within 5 standard errors.
"""
import ctypes
import math

import numpy as np
import pytest
import torch

import bench
from cloudrendering_b200 import _lib, vpt
from oracle import bridge
from tests.harness import SceneSpec, oracle_scene, path_agreement, z_scores

pytestmark = pytest.mark.gpu

GRID, RES, SPP, BOUNCES, SEED = 128, 256, 64, 64, 1
INDEPENDENT_SEED_OFFSET = 0x5BD1E995


class _ModuleCore:
    """Calls C-ABI functions on the module's own context (for the camera matrices)."""

    def __call__(self, name, *args):
        lib = _lib.load()
        ctx = vpt.context_handle()
        _lib.check(getattr(lib, name)(ctx, *args), name, ctx, lib)


def spec(seed_offset=0):
    return SceneSpec(grid=bridge.fbm(GRID, SEED, base_frequency=3.0, contrast=3.5), mode="delta", interp="stochastic",
                     extinction=200.0, albedo=0.99, g=0.85, width=RES, height=RES, env="constant_sun",
                     sky_color=(0.2, 0.2, 0.2), sun_dir=tuple(bench.sun_dir(SEED)), sun_intensity=(5.0, 5.0, 5.0),
                     cam_pos=tuple(bench.camera_pos(SEED)), max_grid_extent=0.5, linear_rgb=1, max_bounces=BOUNCES,
                     fovy=math.radians(60.0), seed_offset=seed_offset)


@pytest.fixture(scope="module")
def module():
    torch.cuda.set_device(0)
    vpt.initialize()
    vpt.set_max_grid_extent(0.5)
    vpt.generate_fbm_cloud(GRID, seed=SEED)
    vpt.set_extinction_scale(200.0)
    vpt.set_scattering_albedo([0.99, 0.99, 0.99])
    vpt.set_phase_g(0.85)
    vpt.set_use_builtin_environment_map("Constant Sky + Sun")
    vpt.set_sky_color([0.2, 0.2, 0.2])
    vpt.set_sun(bench.sun_dir(SEED), [5.0, 5.0, 5.0])
    vpt.set_camera_position(bench.camera_pos(SEED))
    vpt.set_camera_target([0.0, 0.0, 0.0])
    vpt.set_camera_fovy(60.0)
    vpt.set_max_bounces(BOUNCES)
    vpt.set_grid_interpolation("Stochastic")
    vpt.set_vpt_mode_from_name("Delta Tracking")
    vpt.set_denoiser("None")
    vpt.set_seed_offset(0)
    yield vpt
    vpt.cleanup()


def test_grid_is_the_oracle_grid(module):
    lib, ctx = _lib.load(), vpt.context_handle()
    out = np.empty((GRID, GRID, GRID), np.float32)
    _lib.check(lib.vpt_get_dense_grid(ctx, out.ctypes.data_as(ctypes.c_void_p), 0), "grid", ctx, lib)
    assert np.array_equal(out.view(np.uint32), spec().grid.view(np.uint32))


def test_frame0_paths_agree_with_oracle(module):
    img = torch.zeros((4, RES, RES), dtype=torch.float32, device="cuda")
    vpt.set_seed_offset(1)  # a setter clears the accumulation; the next one restores the offset
    vpt.set_seed_offset(0)
    out = vpt.render_frame(img, 1)
    torch.cuda.synchronize()
    got = out[:3].permute(1, 2, 0).cpu().numpy()
    sp = spec()
    sc = oracle_scene(_ModuleCore(), sp, 1)
    ys, xs = np.mgrid[0:RES, 0:RES]
    ref = sc.trace_paths(xs.reshape(-1), ys.reshape(-1), np.zeros(xs.size, np.uint32)).reshape(RES, RES, 3)
    agree = path_agreement(got, ref)
    print(f"config-1 frame 0: path agreement {agree:.5f}")
    assert agree >= 0.99
    assert np.all(out[3].cpu().numpy() == 1.0)


def test_64spp_image_matches_independent_oracle_render(module):
    img = torch.zeros((4, RES, RES), dtype=torch.float32, device="cuda")
    vpt.set_collect_statistics(True)
    vpt.set_seed_offset(1)
    vpt.set_seed_offset(0)
    mean = vpt.render_frame(img, SPP)[:3].permute(1, 2, 0).double().cpu().numpy()
    # the FP64 film and its sum of squares
    s = np.zeros(RES * RES * 3, np.float64)
    sq = np.zeros_like(s)
    _ModuleCore()("vpt_read_statistics", s.ctypes.data_as(ctypes.c_void_p), sq.ctypes.data_as(ctypes.c_void_p), 0,
                  None)
    vpt.set_collect_statistics(False)
    s, sq = s.reshape(RES, RES, 3), sq.reshape(RES, RES, 3)
    assert np.allclose(mean, s / SPP, rtol=1e-6, atol=1e-7)
    sp = spec(INDEPENDENT_SEED_OFFSET)
    sc = oracle_scene(_ModuleCore(), sp, SPP)
    rs, rsq, _ = sc.render(with_sq=True)
    rs, rsq = rs.reshape(s.shape), rsq.reshape(s.shape)
    z = z_scores(s, sq, SPP, rs, rsq, SPP)
    # pixels whose samples are all equal on both sides (sky seen past the cloud): the values must be
    # the same up to float rounding of the per-path radiance
    flat = ~np.isfinite(z)
    ma_px, mb_px = s / SPP, rs / SPP
    assert np.all(np.abs(ma_px - mb_px)[flat] <= 1e-6 * np.abs(mb_px)[flat] + 1e-9)
    zpix = np.abs(np.where(flat, 0.0, z))
    # per-pixel radiance is heavy-tailed (rare paths that see the sun lobe), so the Bonferroni bound is
    # applied to 8x8-pixel bins (4096 samples per bin and side); the pixel-level tail is bounded loosely
    B = 8
    sb = s.reshape(RES // B, B, RES // B, B, 3).sum(axis=(1, 3))
    qb = sq.reshape(RES // B, B, RES // B, B, 3).sum(axis=(1, 3))
    rsb = rs.reshape(RES // B, B, RES // B, B, 3).sum(axis=(1, 3))
    rqb = rsq.reshape(RES // B, B, RES // B, B, 3).sum(axis=(1, 3))
    zb = z_scores(sb, qb, SPP * B * B, rsb, rqb, SPP * B * B)
    zbmax = float(np.nanmax(np.abs(np.where(np.isfinite(zb), zb, 0.0))))
    n = RES * RES * SPP
    ma, mb = s.sum(axis=(0, 1)) / n, rs.sum(axis=(0, 1)) / n
    se = np.sqrt((sq.sum(axis=(0, 1)) / n - ma * ma) / n + (rsq.sum(axis=(0, 1)) / n - mb * mb) / n)
    print(f"config-1 64 spp: binned max |z| {zbmax:.2f}, pixel max |z| {zpix.max():.2f}, pixel |z| > 4: "
          f"{(zpix > 4).mean():.5f}, means {ma} vs {mb}, se {se}")
    assert zbmax < 5.0  # Bonferroni over 32 * 32 * 3 bins
    assert (zpix > 4).mean() < 0.01
    assert np.all(np.abs(ma - mb) <= 1e-3)
    assert np.all(np.abs(ma - mb) <= 5.0 * se)
