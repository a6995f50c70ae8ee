"""The reference's tracker-agreement tests (test/TestVolumetricPathTracing.cpp:156-281) on the CUDA
core, 1:1: 128x128, 64 spp, |mean0 - mean1| <= 1e-3 per RGB channel, the reference's default
medium (extinction 1024, albedo 0.9, g 0.5), default sky with sun lobe, sRGB output, camera at
(0, 0, 0.8), fovy 2 atan(1/2).  Plus the cases the reference does not test (residual ratio
tracking, trilinear, empty-space skipping, the 64-scene-style fBm cloud)."""
import numpy as np
import pytest

from oracle import bridge
from tests.harness import Core, SceneSpec, binned_z, cloud_block, gpu_render, setup_core, z_scores

pytestmark = pytest.mark.gpu

EPS = 1e-3
RES = 128
SPP = 64


@pytest.fixture(scope="module")
def core():
    c = Core(0)
    yield c
    c.close()


def mean_image(core, sp, frames=SPP, sparse=False):
    setup_core(core, sp)
    if sparse:
        core("vpt_set_use_sparse_grid", 1)
    s, sq = gpu_render(core, sp, frames)
    if sparse:
        core("vpt_set_use_sparse_grid", 0)
    return s, sq


def assert_equal_mean(core, sp0, sp1, eps=EPS, frames=SPP, sparse1=False):
    s0, _ = mean_image(core, sp0, frames)
    s1, _ = mean_image(core, sp1, frames, sparse=sparse1)
    m0 = (s0 / frames).mean(axis=(0, 1))
    m1 = (s1 / frames).mean(axis=(0, 1))
    print("means", m0, m1)
    assert np.all(np.abs(m0 - m1) <= eps), (m0, m1)


def spec(grid, mode, **kw):
    return SceneSpec(grid=grid, mode=mode, width=RES, height=RES, **kw)


def test_delta_ratio_equal_mean(core):
    g = cloud_block(1, 1, 1)
    assert_equal_mean(core, spec(g, "delta"), spec(g, "ratio"))


def test_delta_seed_independent_equal_mean(core):
    g = cloud_block(1, 1, 1)
    assert_equal_mean(core, spec(g, "delta"), spec(g, "delta", seed_offset=268435456))


@pytest.mark.parametrize("interp", ["nearest", "stochastic"])
def test_delta_decomposition_equal_mean(core, interp):
    g = cloud_block(8, 8, 8)
    assert_equal_mean(core, spec(g, "delta", interp=interp), spec(g, "decomposition", interp=interp))


def test_delta_decomposition_equal_mean_boundary_layer(core):
    g = cloud_block(8, 8, 8, empty_boundary=True)
    assert_equal_mean(core, spec(g, "delta"), spec(g, "decomposition"))


def test_delta_nee_equal_mean(core):
    g = cloud_block(8, 8, 8, empty_boundary=True)
    assert_equal_mean(core, spec(g, "delta"), spec(g, "nee"))


@pytest.mark.parametrize("size", [1, 8])
def test_delta_dense_sparse_equal_mean(core, size):
    """DeltaTrackingGridTypesGrid1Test / Grid8Test (TestVolumetricPathTracing.cpp:176-196)."""
    g = cloud_block(size, size, size)
    assert_equal_mean(core, spec(g, "delta"), spec(g, "delta"), sparse1=True)


# ---- beyond the reference's suite ----

def fbm_spec(mode, **kw):
    g = bridge.fbm(64, 1, base_frequency=3.0, contrast=3.5)
    base = dict(extinction=200.0, albedo=0.99, g=0.85, env="constant_sun", sky_color=(0.2, 0.2, 0.2),
                sun_dir=(0.3, 0.8, 0.5), sun_intensity=(5.0, 5.0, 5.0), cam_pos=(0.0, 0.3, 2.0),
                max_grid_extent=0.5, linear_rgb=1, fovy=np.radians(60.0), width=96, height=96)
    base.update(kw)
    return SceneSpec(grid=g, mode=mode, **base)


@pytest.mark.parametrize("mode,kw", [("ratio", {}), ("decomposition", {}), ("nee", {}), ("nee", {"use_ess": True}),
                                     ("decomposition", {"interp": "trilinear"}),
                                     ("rrt_unbiased", {"seed_offset": 0x5BD1E995}),
                                     ("rrt_unbiased", {"interp": "trilinear", "seed_offset": 0x5BD1E995}),
                                     ("rrt_unbiased", {"interp": "nearest", "seed_offset": 0x5BD1E995})])
def test_trackers_agree_with_delta_per_pixel(core, mode, kw):
    """Every unbiased tracker agrees with delta tracking on the fBm cloud: per-pixel z-test and the
    image mean within 5 standard errors (NEE's uniform sky sampling of the sun lobe has a heavy
    tail, so a fixed tolerance would not be meaningful)."""
    frames = 128
    base_kw = {k: v for k, v in kw.items() if k == "interp"}
    s0, q0 = mean_image(core, fbm_spec("delta", **base_kw), frames)
    s1, q1 = mean_image(core, fbm_spec(mode, **kw), frames)
    z = z_scores(s0, q0, frames, s1, q1, frames)
    zmax = float(np.nanmax(np.abs(z)))
    zbin, tail = binned_z(s0, q0, frames, s1, q1, frames)
    n = s0.shape[0] * s0.shape[1] * frames
    m0, m1 = s0.sum(axis=(0, 1)) / n, s1.sum(axis=(0, 1)) / n
    se = np.sqrt((q0.sum(axis=(0, 1)) / n - m0 * m0) / n + (q1.sum(axis=(0, 1)) / n - m1 * m1) / n)
    print(mode, kw, "pixel max |z|", zmax, "8x8-bin max |z|", zbin, "pixels |z| > 4", tail, "means", m0, m1, "se", se)
    # Bonferroni over 12 * 12 * 3 bins; next-event estimates (NEE, unbiased RRT) sample the sky
    # uniformly and meet the sun lobe rarely, so their bin means are skewed and the normal tail is
    # optimistic: 5.5 sigma for them
    assert zbin < (5.5 if mode in ("nee", "rrt_unbiased") else 5.0)
    assert tail < 0.01
    assert np.all(np.abs(m0 - m1) <= 5.0 * se)


@pytest.mark.parametrize("mode,prob", [("spectral_delta", 0), ("spectral_delta", 1), ("spectral_delta", 2),
                                       ("spectral_nee", 2)])
def test_spectral_trackers_agree_with_delta_on_grey_media(core, mode, prob):
    """With the same extinction and albedo on every channel, spectral tracking estimates the same
    image as delta tracking (per-pixel z-test and image means)."""
    frames = 128
    # an independent seed: on grey media spectral tracking with the same seeds retraces delta
    # tracking's paths almost exactly, and a z-test needs independent estimates
    s0, q0 = mean_image(core, fbm_spec("delta"), frames)
    s1, q1 = mean_image(core, fbm_spec(mode, sdt_prob=prob, seed_offset=0x5BD1E995), frames)
    z = z_scores(s0, q0, frames, s1, q1, frames)
    zmax = float(np.nanmax(np.abs(z)))
    zbin, tail = binned_z(s0, q0, frames, s1, q1, frames)
    n = s0.shape[0] * s0.shape[1] * frames
    m0, m1 = s0.sum(axis=(0, 1)) / n, s1.sum(axis=(0, 1)) / n
    se = np.sqrt((q0.sum(axis=(0, 1)) / n - m0 * m0) / n + (q1.sum(axis=(0, 1)) / n - m1 * m1) / n)
    print(mode, prob, "pixel max |z|", zmax, "8x8-bin max |z|", zbin, "pixels |z| > 4", tail, "means", m0, m1,
          "se", se)
    assert zbin < (5.5 if mode == "spectral_nee" else 5.0)  # as above
    assert tail < 0.01
    assert np.all(np.abs(m0 - m1) <= 5.0 * se)


def test_spectral_delta_chromatic_extinction_matches_per_channel_delta(core):
    """Chromatic media: each channel of spectral delta tracking equals delta tracking of a grey
    medium with that channel's extinction (image means within 5 standard errors)."""
    frames = 128
    ext = (1.0, 0.55, 0.3)
    s1, q1 = mean_image(core, fbm_spec("spectral_delta", extinction_base=ext, sdt_prob=2), frames)
    n = s1.shape[0] * s1.shape[1] * frames
    m1 = s1.sum(axis=(0, 1)) / n
    v1 = q1.sum(axis=(0, 1)) / n - m1 * m1
    for c in range(3):
        s0, q0 = mean_image(core, fbm_spec("delta", extinction_base=(ext[c],) * 3), frames)
        m0 = s0.sum(axis=(0, 1))[c] / n
        v0 = q0.sum(axis=(0, 1))[c] / n - m0 * m0
        se = np.sqrt(v0 / n + v1[c] / n)
        print("channel", c, m0, m1[c], se)
        assert abs(m0 - m1[c]) <= 5.0 * se


def test_delta_unbiased_residual_ratio_equal_mean(core):
    """The reference suite's equal-mean check on its 8^3 block with the empty boundary layer (128^2,
    64 spp) for the unbiased residual ratio tracker.  Its estimate has about ten times delta tracking's
    standard error on this fixture (one supervoxel holds the block and the empty layer, so the control
    extinction lies between them and the ratio factors reach 1.42), so the bound is 5 standard errors
    of the difference instead of 1e-3."""
    g = cloud_block(8, 8, 8, empty_boundary=True)
    s0, q0 = mean_image(core, spec(g, "delta"))
    s1, q1 = mean_image(core, spec(g, "rrt_unbiased", seed_offset=0x5BD1E995))
    n = RES * RES * SPP
    m0, m1 = s0.sum(axis=(0, 1)) / n, s1.sum(axis=(0, 1)) / n
    se = np.sqrt((q0.sum(axis=(0, 1)) / n - m0 * m0) / n + (q1.sum(axis=(0, 1)) / n - m1 * m1) / n)
    print("delta", m0, "unbiased residual ratio", m1, "se", se)
    assert np.all(np.abs(m0 - m1) <= 5.0 * se)


def test_reference_residual_ratio_estimator_is_biased(core):
    """The reference's residual ratio tracking (ResidualRatioTracking.glsl, marked work in progress
    upstream) does not estimate the same image as delta tracking.  The core reproduces it path for
    path (test_gpu_parity); this test pins the size of the deviation on the fBm scene (the oracle
    gives -0.064, -9 standard errors: mean 0.208 against 0.272), which the unbiased tracker above
    does not show."""
    frames = 64
    s0, q0 = mean_image(core, fbm_spec("delta"), frames)
    s1, q1 = mean_image(core, fbm_spec("rrt"), frames)
    n = s0.shape[0] * s0.shape[1] * frames
    m0, m1 = s0.sum(axis=(0, 1)) / n, s1.sum(axis=(0, 1)) / n
    se = np.sqrt((q0.sum(axis=(0, 1)) / n - m0 * m0) / n + (q1.sum(axis=(0, 1)) / n - m1 * m1) / n)
    print("reference residual ratio tracking vs delta:", m1, m0, "se", se)
    assert np.all(np.isfinite(m1))
    assert np.all(m0 - m1 > 5.0 * se)
