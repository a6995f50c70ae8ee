"""CPU tests of the oracle itself: the reference's own tracker-agreement tests
(test/TestVolumetricPathTracing.cpp:156-281) run on the oracle at reduced size, plus properties of
the scene and acceleration-structure builders."""
import math

import numpy as np
import pytest

from oracle import bridge
from tests.harness import SceneSpec, cloud_block, oracle_scene, z_scores


def render(sp, frames, threads=0):
    sc = oracle_scene(None, sp, frames)
    film, sq, lookups = sc.render(threads=threads, with_sq=True)
    shape = (sp.height, sp.width, 3)
    return film.reshape(shape), sq.reshape(shape), lookups


def assert_equal_mean(sp0, sp1, frames, zmax=5.0):
    """Image means agree within 5 standard errors of the difference, and the per-pixel z-test
    (Bonferroni at alpha = 1e-3 over all pixels) passes."""
    s0, q0, _ = render(sp0, frames)
    s1, q1, _ = render(sp1, frames)
    z = z_scores(s0, q0, frames, s1, q1, frames)
    assert np.nanmax(np.abs(z)) < 6.0, np.nanmax(np.abs(z))
    m0, m1 = s0 / frames, s1 / frames
    n = m0.shape[0] * m0.shape[1]
    v0 = np.maximum(q0 / frames - m0 * m0, 0).sum(axis=(0, 1)) / (frames * n * n)
    v1 = np.maximum(q1 / frames - m1 * m1, 0).sum(axis=(0, 1)) / (frames * n * n)
    diff = np.abs(m0.mean(axis=(0, 1)) - m1.mean(axis=(0, 1)))
    assert np.all(diff <= zmax * np.sqrt(v0 + v1) + 1e-9), (diff, np.sqrt(v0 + v1))


W, F = 40, 24


def test_delta_ratio_equal_mean_block1():
    g = cloud_block(1, 1, 1)
    assert_equal_mean(SceneSpec(g, "delta", width=W, height=W), SceneSpec(g, "ratio", width=W, height=W), F)


def test_delta_seed_independent_equal_mean():
    g = cloud_block(1, 1, 1)
    assert_equal_mean(SceneSpec(g, "delta", width=W, height=W),
                      SceneSpec(g, "delta", width=W, height=W, seed_offset=268435456), F)


@pytest.mark.parametrize("interp", ["nearest", "stochastic"])
def test_delta_decomposition_equal_mean_block8(interp):
    g = cloud_block(8, 8, 8)
    assert_equal_mean(SceneSpec(g, "delta", interp=interp, width=W, height=W),
                      SceneSpec(g, "decomposition", interp=interp, width=W, height=W), F)


def test_delta_decomposition_equal_mean_boundary_layer():
    g = cloud_block(8, 8, 8, empty_boundary=True)
    assert_equal_mean(SceneSpec(g, "delta", width=W, height=W), SceneSpec(g, "decomposition", width=W, height=W), F)


def test_delta_nee_equal_mean_boundary_layer():
    g = cloud_block(8, 8, 8, empty_boundary=True)
    assert_equal_mean(SceneSpec(g, "delta", width=W, height=W), SceneSpec(g, "nee", width=W, height=W), F)


def test_nee_with_empty_space_skipping_equal_mean():
    g = bridge.fbm(24, 3)
    kw = dict(extinction=200.0, width=W, height=W)
    assert_equal_mean(SceneSpec(g, "nee", **kw), SceneSpec(g, "nee", use_ess=True, **kw), F)


def test_trilinear_decomposition_equal_mean():
    g = bridge.fbm(16, 5)
    kw = dict(interp="trilinear", extinction=300.0, width=W, height=W)
    assert_equal_mean(SceneSpec(g, "delta", **kw), SceneSpec(g, "decomposition", **kw), F)


def test_bounce_cap_darkens_only():
    g = cloud_block(8, 8, 8)
    s0, _, _ = render(SceneSpec(g, "delta", width=24, height=24), 8)
    s1, _, _ = render(SceneSpec(g, "delta", width=24, height=24, max_bounces=1), 8)
    assert np.all(s1 <= s0 + 1e-12)
    assert s1.sum() < s0.sum()


def test_rng_stream_is_deterministic_and_in_range():
    a, st_a = bridge.rng_stream(12345, 1000)
    b, st_b = bridge.rng_stream(12345, 1000)
    assert np.array_equal(a, b) and np.array_equal(st_a, st_b)
    assert a.min() >= 0.0 and a.max() <= 1.0
    assert abs(a.mean() - 0.5) < 0.03


def test_fbm_cloud_statistics():
    g = bridge.fbm(64, 1, base_frequency=3.0, contrast=3.5)
    empty = (g == 0).mean()
    assert 0.30 < empty < 0.40, empty  # config: ~35% empty after clamping values < 0.3
    assert g.max() <= 1.0 and g[g > 0].min() >= 0.3
    assert np.array_equal(g, bridge.fbm(64, 1, base_frequency=3.0, contrast=3.5))
    assert not np.array_equal(g, bridge.fbm(64, 2, base_frequency=3.0, contrast=3.5))


def test_supervoxel_stats_properties():
    g = cloud_block(8, 8, 8)
    mn, mx, avg, occ = bridge.supervoxel_stats(g, 8, 0)
    assert mn.tolist() == [1.0] and mx.tolist() == [1.0] and avg.tolist() == [1.0] and occ.tolist() == [1]
    mn, mx, avg, occ = bridge.supervoxel_stats(g, 8, 1)  # halo reaches the zero border
    assert mn.tolist() == [0.0] and mx.tolist() == [1.0]
    assert avg[0] == np.float32(512.0 / 1000.0)
    g = cloud_block(12, 8, 8)  # partial boundary supervoxel along x -> min forced to 0
    mn, mx, avg, occ = bridge.supervoxel_stats(g, 8, 0)
    assert mn.tolist() == [1.0, 0.0]
    e = np.zeros((16, 16, 16), np.float32)
    e[3, 3, 3] = 1e-6
    mn, mx, avg, occ = bridge.supervoxel_stats(e, 8, 0)
    assert occ.tolist() == [0] * 8  # max < 1e-5 counts as empty


def test_occupancy_halo():
    g = np.zeros((16, 16, 16), np.float32)
    g[8, 8, 8] = 0.5  # voxel in block (1,1,1)
    assert bridge.occupancy(g, 8, 0).sum() == 1
    assert bridge.occupancy(g, 8, 1).sum() == 8  # halo touches all 8 blocks around the corner


def test_eaw_constant_image_is_fixed_point():
    c = np.full((32, 32, 4), 0.25, np.float32)
    out = bridge.eaw(c, None, None, 3)
    assert np.allclose(out, 0.25, atol=1e-7)
    noisy = np.random.default_rng(0).random((32, 32, 4)).astype(np.float32)
    out = bridge.eaw(noisy, None, None, 3)
    assert out.std() < noisy.std()


def test_env_pyramid_of_constant_image():
    rgba = np.ones((16, 32, 4), np.float32)
    rgba[..., :3] = 0.5
    pyr = bridge.env_pyramid(rgba, 4)
    assert np.allclose(pyr, math.sqrt(3) * 0.5, rtol=1e-6)
