"""GPU parity tests: the CUDA core (through its C ABI) against the CPU oracle on the same inputs.

* integer / builder work is bit-exact: fBm grid, supervoxel min/max/mean/occupancy, occupancy grid;
* paths: every camera path of a 1-spp frame is traced by both sides from the same seed and camera
  matrix; they take the same random decisions, so the radiance agrees to float rounding except for
  paths where a libm / CUDA transcendental differs by an ulp and flips a later comparison.  The test
  requires >= 99% of paths to agree to rtol 1e-4 (measured agreement is printed);
* images: per-pixel z-test (Bonferroni, |z| < 6) and image-mean agreement at 64 frames.
"""
import ctypes

import numpy as np
import pytest
import torch

from oracle import bridge
from tests.harness import (Core, SceneSpec, cloud_block, gpu_render, oracle_scene, path_agreement, setup_core,
                           z_scores)

pytestmark = pytest.mark.gpu

AGREE_MIN = 0.99


@pytest.fixture(scope="module")
def core():
    c = Core(0)
    yield c
    c.close()


def dptr(t: torch.Tensor):
    return ctypes.c_void_p(t.data_ptr())


def test_fbm_grid_bit_exact(core):
    for (nx, ny, nz), seed in [((64, 64, 64), 1), ((40, 24, 33), 7)]:
        core("vpt_generate_fbm_grid", nx, ny, nz, seed, 6, 2.0, 0.5, 3.0, 0.3)
        out = np.empty((nz, ny, nx), np.float32)
        core("vpt_get_dense_grid", out.ctypes.data_as(ctypes.c_void_p), 0)
        ref = bridge.fbm((nx, ny, nz), seed, base_frequency=3.0, contrast=3.5)
        assert np.array_equal(out.view(np.uint32), ref.view(np.uint32))


@pytest.mark.parametrize("shape,sv,halo", [((64, 64, 64), 8, 0), ((64, 64, 64), 8, 1), ((37, 20, 29), 8, 1),
                                           ((6, 6, 6), 2, 0)])
def test_supervoxel_grid_bit_exact(core, shape, sv, halo):
    nz, ny, nx = shape
    g = bridge.fbm((nx, ny, nz), 11, base_frequency=3.0, contrast=3.5)
    d = torch.from_numpy(g).cuda()
    gx, gy, gz = -(-nx // sv), -(-ny // sv), -(-nz // sv)
    n = gx * gy * gz
    mn, mx, avg = (torch.empty(n, device="cuda") for _ in range(3))
    occ = torch.empty(n, dtype=torch.uint8, device="cuda")
    lib = core.lib
    assert lib.vpt_build_supervoxel_grid(dptr(d), nx, ny, nz, sv, halo, dptr(mn), dptr(mx), dptr(avg), dptr(occ),
                                         None) == 0
    torch.cuda.synchronize()
    rmn, rmx, ravg, rocc = bridge.supervoxel_stats(g, sv, halo)
    assert np.array_equal(mn.cpu().numpy().view(np.uint32), rmn.view(np.uint32))
    assert np.array_equal(mx.cpu().numpy().view(np.uint32), rmx.view(np.uint32))
    assert np.array_equal(avg.cpu().numpy().view(np.uint32), ravg.view(np.uint32))
    assert np.array_equal(occ.cpu().numpy(), rocc)
    pairs = torch.empty(2 * n, device="cuda")
    assert lib.vpt_build_rrt_params(dptr(mn), dptr(mx), dptr(avg), n, 1000.0, sv, dptr(pairs), None) == 0
    torch.cuda.synchronize()
    ref = bridge.rrt_params(rmn, rmx, ravg, 1000.0, sv)
    # mu_c uses powf (CUDA vs libm may differ by one ulp); mu_r_bar is exact
    got = pairs.cpu().numpy()
    assert np.array_equal(got[1::2], ref[1::2])
    assert np.allclose(got[0::2], ref[0::2], rtol=2e-7, atol=0)


@pytest.mark.parametrize("key", sorted(__import__("tests.harness", fromlist=["_"]).supervoxel_golden()))
def test_supervoxel_grid_matches_reference_builder(core, key):
    """The core's supervoxel builders against SuperVoxelGrid.cpp compiled unmodified (fixture
    tests/golden/supervoxel_grids.npz): min / max / occupancy bit for bit, mu_r_bar bit for bit, mu_c to
    one ulp (powf)."""
    from tests.harness import supervoxel_golden, supervoxel_size

    g = supervoxel_golden()[key]
    raw = g["raw"]
    nz, ny, nx = raw.shape
    sv = supervoxel_size(nx, ny, nz)
    vmin, vmax = bridge.minmax(raw)
    d = torch.from_numpy(bridge.normalize(raw, vmin, vmax)).cuda()
    n = g["occ_rrt"].size
    mn, mx, avg = (torch.empty(n, device="cuda") for _ in range(3))
    occ = torch.empty(n, dtype=torch.uint8, device="cuda")
    lib = core.lib
    halo = 0 if g["interp"] == 0 else 1
    assert lib.vpt_build_supervoxel_grid(dptr(d), nx, ny, nz, sv, halo, dptr(mn), dptr(mx), dptr(avg), dptr(occ),
                                         None) == 0
    pairs = torch.empty(2 * n, device="cuda")
    assert lib.vpt_build_rrt_params(dptr(mn), dptr(mx), dptr(avg), n, g["extinction"], sv, dptr(pairs), None) == 0
    torch.cuda.synchronize()
    assert np.array_equal(mn.cpu().numpy().view(np.uint32), g["minmax"][0::2].view(np.uint32))
    assert np.array_equal(mx.cpu().numpy().view(np.uint32), g["minmax"][1::2].view(np.uint32))
    assert np.array_equal(occ.cpu().numpy(), g["occ_decomposition"])
    got = pairs.cpu().numpy()
    assert np.array_equal(got[1::2].view(np.uint32), g["rrt"][1::2].view(np.uint32))
    assert np.allclose(got[0::2], g["rrt"][0::2], rtol=2e-7, atol=0)


def test_residual_ratio_grid_bit_exact(core):
    """The unbiased residual ratio tracker's supervoxel grid: (mu_c, mu_r_bar) as the reference's
    formulas (mu_c through powf: one ulp allowed), the majorant reciprocals bit-exact."""
    g = bridge.fbm((64, 48, 40), 13, base_frequency=3.0, contrast=3.5)
    g[:8, :8, :8] = 0.0  # an empty supervoxel (its halo reaches the neighbours: one corner cell)
    nz, ny, nx = g.shape
    d = torch.from_numpy(g).cuda()
    sv = 8
    n = (-(-nx // sv)) * (-(-ny // sv)) * (-(-nz // sv))
    mn, mx, avg = (torch.empty(n, device="cuda") for _ in range(3))
    occ = torch.empty(n, dtype=torch.uint8, device="cuda")
    lib = core.lib
    assert lib.vpt_build_supervoxel_grid(dptr(d), nx, ny, nz, sv, 1, dptr(mn), dptr(mx), dptr(avg), dptr(occ),
                                         None) == 0
    out = torch.empty(4 * n, device="cuda")
    assert lib.vpt_build_residual_ratio_grid(dptr(mn), dptr(mx), dptr(avg), n, 700.0, sv, dptr(out), None) == 0
    torch.cuda.synchronize()
    rmn, rmx, ravg, _ = bridge.supervoxel_stats(g, sv, 1)
    ref = bridge.rrt_local(rmn, rmx, ravg, 700.0, sv).reshape(-1, 4)
    got = out.cpu().numpy().reshape(-1, 4)
    assert np.array_equal(got[:, 1:].view(np.uint32), ref[:, 1:].view(np.uint32))
    assert np.allclose(got[:, 0], ref[:, 0], rtol=2e-7, atol=0)
    assert (got[:, 3] == 0).any() and (got[:, 3] > 0).any()


@pytest.mark.parametrize("halo", [0, 1])
def test_occupancy_grid_bit_exact(core, halo):
    g = bridge.fbm((48, 40, 56), 3, base_frequency=3.0, contrast=3.5)
    g[g < 0.6] = 0.0
    nz, ny, nx = g.shape
    d = torch.from_numpy(g).cuda()
    n = 6 * 5 * 7
    out = torch.empty(n, dtype=torch.uint8, device="cuda")
    assert core.lib.vpt_build_occupancy_grid(dptr(d), nx, ny, nz, 8, halo, 0.0, dptr(out), None) == 0
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), bridge.occupancy(g, 8, halo, 0.0))


def test_environment_pyramid_matches_oracle(core):
    rng = np.random.default_rng(4)
    rgba = np.ones((32, 64, 4), np.float32)
    rgba[..., :3] = rng.random((32, 64, 3)).astype(np.float32) * 3.0
    levels = 8
    total = sum((1 << (levels - l)) ** 2 for l in range(levels))
    d = torch.from_numpy(rgba).cuda()
    out = torch.empty(total, device="cuda")
    assert core.lib.vpt_build_environment_pyramid(dptr(d), 64, 32, levels, dptr(out), None) == 0
    torch.cuda.synchronize()
    ref = bridge.env_pyramid(rgba, levels)
    assert np.allclose(out.cpu().numpy(), ref, rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize("quirk", [0, 1])
def test_eaw_matches_oracle(core, quirk):
    rng = np.random.default_rng(5)
    h, w = 48, 64
    color = rng.random((h, w, 4)).astype(np.float32)
    pos = rng.random((h, w, 4)).astype(np.float32) * 0.2
    nrm = rng.random((h, w, 4)).astype(np.float32)
    dc, dp, dn = (torch.from_numpy(a).cuda() for a in (color, pos, nrm))
    out = torch.empty_like(dc)
    assert core.lib.vpt_eaw_denoise_rgba(dptr(dc), dptr(dp), dptr(dn), w, h, 3, 5.0, 0.1, 0.1, quirk, dptr(out),
                                         None) == 0
    torch.cuda.synchronize()
    ref = bridge.eaw(color, pos, nrm, 3, 5.0, 0.1, 0.1, quirk)
    assert np.allclose(out.cpu().numpy(), ref, rtol=1e-5, atol=1e-6)


def test_density_texture_follows_a_new_grid_and_a_nonzero_border(core_dr):
    """The texture array is kept for grids of the same size and refilled for each new grid: a second
    grid rendered on the same context gives the film of a fresh context (the first grid's texels are
    gone).  A grid whose minimum is above 0 has a non-zero border density, which the texture's border
    colour cannot represent: it is read by global loads, with the same film as with the option off."""
    core = core_dr
    a = fbm_scene(width=32, height=32, mode="delta")
    b = fbm_scene(width=32, height=32, mode="delta", grid=bridge.fbm(48, 9, base_frequency=2.0, contrast=6.0))
    setup_core(core, a)
    gpu_render(core, a, 2, stats=False)
    setup_core(core, b)  # same 48^3 size: the array is reused
    s_reused, _ = gpu_render(core, b, 2, stats=False)
    fresh = Core(0, "dr")
    try:
        setup_core(fresh, b)
        s_fresh, _ = gpu_render(fresh, b, 2, stats=False)
    finally:
        fresh.close()
    assert np.allclose(s_reused, s_fresh, rtol=1e-12, atol=1e-12)
    # minimum 0.25 everywhere: border density (0 - 0.25) / 0.75 != 0
    g = (0.25 + 0.75 * np.asarray(b.grid, np.float32)).astype(np.float32)
    c = fbm_scene(width=32, height=32, mode="delta", grid=g)
    setup_core(core, c)
    films = []
    for tex in (1.0, 0.0):
        core("vpt_set_option", b"density_texture", tex)
        films.append(gpu_render(core, c, 2, stats=False)[0])
    core("vpt_set_option", b"density_texture", 1.0)
    assert np.allclose(films[0], films[1], rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("size", [(64, 48), (37, 50), (300, 200)])
def test_eaw_lattice_tiles_equal_direct_taps(core, size):
    """The shared-memory EAW pass (taps of 16 x 16 pixels of one residue class staged per block) gives
    exactly the image of the pass that reads every tap from global memory, for ragged image sizes and
    every step up to 16."""
    w, h = size
    sp = fbm_scene(width=w, height=h, mode="delta")
    setup_core(core, sp)
    core("vpt_set_denoiser", 1)
    core("vpt_set_denoiser_property", b"iterations", b"5")
    core("vpt_render_frames", 4, None)
    outs = []
    for lattice in (b"1", b"0"):
        core("vpt_set_denoiser_property", b"lattice_tiles", lattice)
        o = np.zeros(4 * w * h, np.float32)
        core("vpt_read_result", o.ctypes.data_as(ctypes.c_void_p), 4, 0, None)
        outs.append(o)
    core("vpt_set_denoiser_property", b"lattice_tiles", b"1")
    core("vpt_set_denoiser", 0)
    assert np.all(np.isfinite(outs[0]))
    assert np.array_equal(outs[0], outs[1])


def test_eaw_rejects_an_output_that_overlaps_an_input(core):
    h, w = 16, 16
    imgs = [torch.rand((h, w, 4), device="cuda") for _ in range(3)]
    for out in (imgs[0], imgs[1], imgs[2], imgs[0][3:]):
        st = core.lib.vpt_eaw_denoise_rgba(dptr(imgs[0]), dptr(imgs[1]), dptr(imgs[2]), w, h, 3, 5.0, 0.1, 0.1, 0,
                                           dptr(out), None)
        assert st == 1  # VPT_ERR_ARG
    torch.cuda.synchronize()


def fbm_scene(**kw):
    g = bridge.fbm(48, 2, base_frequency=3.0, contrast=3.5)
    base = dict(grid=g, extinction=150.0, albedo=0.99, g=0.85, width=64, height=64, env="constant_sun",
                sky_color=(0.2, 0.2, 0.2), sun_dir=(0.3, 0.8, 0.5), sun_intensity=(5.0, 5.0, 5.0),
                cam_pos=(0.3, 0.4, 1.4), max_grid_extent=0.5, linear_rgb=1, max_bounces=64)
    base.update(kw)
    return SceneSpec(**base)


PATH_CASES = {
    "delta_stochastic": dict(mode="delta"),
    "delta_nearest": dict(mode="delta", interp="nearest"),
    "delta_trilinear": dict(mode="delta", interp="trilinear"),
    "ratio": dict(mode="ratio"),
    "nee": dict(mode="nee"),
    "nee_ess": dict(mode="nee", use_ess=True),
    "decomposition": dict(mode="decomposition"),
    "decomposition_trilinear": dict(mode="decomposition", interp="trilinear"),
    "rrt": dict(mode="rrt"),
    # the unbiased residual ratio tracker (no reference counterpart): every interpolation, lights
    "rrt_unbiased": dict(mode="rrt_unbiased"),
    "rrt_unbiased_nearest": dict(mode="rrt_unbiased", interp="nearest"),
    "rrt_unbiased_trilinear": dict(mode="rrt_unbiased", interp="trilinear"),
    "rrt_unbiased_lights": dict(mode="rrt_unbiased", lights=[
        dict(type="Point Light", space="World", position=(0.6, 0.8, 0.3), intensity=0.8, color=(1.0, 0.8, 0.6))]),
    "delta_default_sky": dict(mode="delta", env="default", linear_rgb=0),
    "nee_default_sky_g0": dict(mode="nee", env="default", g=0.0),
    # lights of the light editor: a view-space spot light and a world-space point light; a
    # directional light under a black sky (all NEE samples go to the light)
    "nee_lights": dict(mode="nee", lights=[
        dict(type="Spotlight", space="View", position=(0.05, 0.1, 0.0), spot_direction=(0.0, -0.1, -1.0),
             spot_total_width=0.6, spot_falloff_start=0.3, intensity=3.0),
        dict(type="Point Light", space="World", position=(0.6, 0.8, 0.3), intensity=0.8, color=(1.0, 0.8, 0.6))]),
    "nee_light_directional_black": dict(mode="nee", env="black", lights=[
        dict(type="Directional Light", space="View Orientation", position=(0.4, 0.9, 0.2), intensity=2.0)]),
    # escape radiance depends on the direction and paths are not capped: a diverged path shows
    "delta_default_sky_linear_uncapped": dict(mode="delta", env="default", linear_rgb=1, max_bounces=0),
    "decomposition_default_sky_uncapped": dict(mode="decomposition", env="default", linear_rgb=1, max_bounces=0),
    "rrt_default_sky_uncapped": dict(mode="rrt", env="default", linear_rgb=1, max_bounces=0),
    # spectral trackers: chromatic extinction and albedo, each collision-probability mode
    "spectral_delta_max": dict(mode="spectral_delta", sdt_prob=0, extinction_base=(1.0, 0.55, 0.3),
                               albedo_rgb=(0.99, 0.9, 0.8)),
    "spectral_delta_avg": dict(mode="spectral_delta", sdt_prob=1, extinction_base=(1.0, 0.55, 0.3),
                               albedo_rgb=(0.99, 0.9, 0.8)),
    "spectral_delta_hist": dict(mode="spectral_delta", sdt_prob=2, extinction_base=(0.4, 1.0, 0.7),
                                albedo_rgb=(0.95, 0.99, 0.9)),
    "spectral_delta_hist_trilinear": dict(mode="spectral_delta", sdt_prob=2, interp="trilinear",
                                          extinction_base=(1.0, 0.55, 0.3), albedo_rgb=(0.99, 0.9, 0.8)),
    "spectral_nee_hist": dict(mode="spectral_nee", sdt_prob=2, extinction_base=(1.0, 0.55, 0.3),
                              albedo_rgb=(0.99, 0.9, 0.8)),
    "spectral_nee_max_ess": dict(mode="spectral_nee", sdt_prob=0, use_ess=True, extinction_base=(1.0, 0.55, 0.3),
                                 albedo_rgb=(0.99, 0.9, 0.8)),
    "spectral_nee_lights": dict(mode="spectral_nee", sdt_prob=2, extinction_base=(1.0, 0.55, 0.3),
                                albedo_rgb=(0.99, 0.9, 0.8), lights=[
        dict(type="Point Light", space="World", position=(0.6, 0.8, 0.3), intensity=0.8, color=(1.0, 0.8, 0.6))]),
}


@pytest.fixture(scope="module")
def core_dr():
    c = Core(0, "dr")
    yield c
    c.close()


@pytest.mark.parametrize("case", sorted(PATH_CASES))
@pytest.mark.parametrize("variant", ["default", "dr"])
def test_path_parity(core, core_dr, case, variant):
    """Every path of a 1-spp frame, CUDA core against the oracle.  ``dr``: both sides evaluate
    transcendentals in double precision rounded to float, and every path must agree."""
    c = core if variant == "default" else core_dr
    sp = fbm_scene(**PATH_CASES[case])
    setup_core(c, sp)
    s, _ = gpu_render(c, sp, 1, stats=False)
    sc = oracle_scene(c, sp, 1)
    ys, xs = np.mgrid[0:sp.height, 0:sp.width]
    with bridge.double_rounded_math(variant == "dr"):
        ref = sc.trace_paths(xs.reshape(-1), ys.reshape(-1), np.zeros(xs.size, np.uint32)).reshape(
            sp.height, sp.width, 3)
    agree = path_agreement(s.astype(np.float32), ref)
    print(f"[{variant}] {case}: path agreement {agree:.5f}")
    assert agree >= (AGREE_MIN if variant == "default" else 0.999)


def test_path_parity_environment_image(core):
    rng = np.random.default_rng(9)
    rgba = np.ones((64, 128, 4), np.float32)
    rgba[..., :3] = 0.2
    rgba[10:14, 40:46, :3] = 50.0  # a small bright "sun" patch
    rgba[..., :3] += rng.random((64, 128, 3)).astype(np.float32) * 0.05
    sp = fbm_scene(mode="nee", env="image", env_rgba=rgba)
    setup_core(core, sp)
    s, _ = gpu_render(core, sp, 1, stats=False)
    sc = oracle_scene(core, sp, 1)
    ys, xs = np.mgrid[0:sp.height, 0:sp.width]
    ref = sc.trace_paths(xs.reshape(-1), ys.reshape(-1), np.zeros(xs.size, np.uint32)).reshape(sp.height, sp.width, 3)
    agree = path_agreement(s.astype(np.float32), ref)
    print(f"env image nee: path agreement {agree:.5f}")
    assert agree >= AGREE_MIN


@pytest.mark.parametrize("case", ["delta_stochastic", "nee", "decomposition", "rrt", "rrt_unbiased"])
def test_image_statistics_match_oracle(core, case):
    sp = fbm_scene(**PATH_CASES[case], width=48, height=48)
    frames = 64
    setup_core(core, sp)
    s, sq = gpu_render(core, sp, frames)
    sc = oracle_scene(core, sp, frames)
    rs, rsq, _ = sc.render(with_sq=True)
    rs = rs.reshape(s.shape)
    rsq = rsq.reshape(s.shape)
    z = z_scores(s, sq, frames, rs, rsq, frames)
    assert np.nanmax(np.abs(z)) < 6.0
    assert np.all(np.abs(s.mean(axis=(0, 1)) - rs.mean(axis=(0, 1))) / frames <= 1e-3)


def test_lookup_counter_matches_oracle(core):
    sp = fbm_scene(mode="delta", width=32, height=32)
    setup_core(core, sp)
    core("vpt_reset_stats")
    gpu_render(core, sp, 4, stats=False)
    from cloudrendering_b200._lib import VptStats
    st = VptStats()
    core("vpt_get_stats", ctypes.byref(st))
    sc = oracle_scene(core, sp, 4)
    _, _, lookups = sc.render()
    assert st.paths == 32 * 32 * 4
    assert abs(st.density_lookups - lookups) <= 0.01 * lookups


def test_iteration_guard_reports_error_without_hanging(core):
    sp = SceneSpec(grid=cloud_block(8, 8, 8), mode="delta", width=16, height=16)
    setup_core(core, sp)
    core("vpt_reset_stats")
    core("vpt_set_option", b"max_steps_per_path", 8.0)
    core("vpt_render_frames", 1, None)
    st = core.lib.vpt_synchronize(core.ctx, None)
    assert st == 4  # VPT_ERR_ITER_LIMIT
    core("vpt_set_option", b"max_steps_per_path", float(1 << 24))
    core("vpt_reset_stats")
    core("vpt_render_frames", 1, None)
    core("vpt_synchronize", None)


@pytest.mark.parametrize("mode", ["delta", "ratio", "nee", "nee_lights", "delta_isosurfaces",
                                  "delta_isosurfaces_gradient", "delta_isosurfaces_cook_torrance", "nee_ess",
                                  "nee_ess_ref_compat", "decomposition", "decomposition_trilinear", "rrt_unbiased",
                                  "rrt_unbiased_trilinear", "rrt_unbiased_lights"])
def test_schedules_trace_identical_paths(core_dr, mode):
    """Tile, persistent-batch and per-lane-refill schedules trace the same paths (same film up to the
    order of the FP64 atomic additions).  The isosurface case covers the refill loop's own surface
    handling (iteration cap, weight cut-off, per-lane reset of the surface state).  On the parity
    build, whose operations are not contracted: the product build may contract the refill loop's and
    the recursive trackers' expressions differently."""
    core = core_dr
    if mode == "nee_lights":
        kw = PATH_CASES["nee_lights"]
    elif mode == "delta_isosurfaces":
        kw = dict(mode="delta", interp="trilinear", iso=True, iso_value=0.3)
    elif mode == "delta_isosurfaces_gradient":
        kw = dict(mode="delta", interp="trilinear", iso=True, iso_value=0.02, iso_type="Gradient")
    elif mode == "delta_isosurfaces_cook_torrance":
        kw = dict(mode="delta", interp="trilinear", iso=True, iso_value=0.3, iso_brdf="Cook Torrance",
                  brdf_params={"metallic": 0.5, "roughness": 0.3})
    elif mode.startswith("nee_ess"):  # sky shadow rays skip empty occupancy blocks (the refill loop's own walk)
        kw = dict(mode="nee", use_ess=True, ess_ref_compat=mode.endswith("compat"))
    elif mode == "rrt_unbiased_lights":  # free flights and shadow walks of the refill loop, light shadow rays
        kw = dict(PATH_CASES["nee_lights"], mode="rrt_unbiased")
    elif mode.startswith("rrt_unbiased"):
        kw = dict(mode="rrt_unbiased", interp="trilinear" if mode.endswith("trilinear") else "stochastic")
    elif mode.startswith("decomposition"):  # the supervoxel walk with two clocks in the refill loop
        kw = dict(mode="decomposition", interp="trilinear" if mode.endswith("trilinear") else "stochastic")
    else:
        kw = dict(mode=mode)
    sp = fbm_scene(width=40, height=40, **kw)
    setup_core(core, sp)
    core("vpt_set_option", b"ess_ref_compat", 1.0 if sp.ess_ref_compat else 0.0)
    films = []
    for sched in (0, 1, 2):
        core("vpt_set_option", b"schedule", float(sched))
        s, _ = gpu_render(core, sp, 3, stats=False)
        films.append(s)
    # refills taken as soon as one lane waits, or once 8 wait (the default is 4): the same paths
    for k in (1.0, 8.0):
        core("vpt_set_option", b"refill_min_lanes", k)
        films.append(gpu_render(core, sp, 3, stats=False)[0])
    core("vpt_set_option", b"refill_min_lanes", 4.0)
    core("vpt_set_option", b"schedule", 2.0)
    core("vpt_set_option", b"ess_ref_compat", 0.0)
    for f in films[1:]:
        assert np.allclose(films[0], f, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("interp", ["nearest", "stochastic", "trilinear"])
@pytest.mark.parametrize("sched", [1, 2])
@pytest.mark.parametrize("mode", ["delta", "ratio", "nee", "nee_ess", "decomposition", "rrt_unbiased"])
def test_density_texture_reads_the_same_texels(core_dr, interp, sched, mode):
    """Delta, ratio and next event tracking through the grid's 3D texture object (option
    density_texture) trace the same paths as through global loads: same film (up to the order of the
    FP64 additions) and the same feature maps, in the persistent and per-lane refill schedules, for
    every interpolation, with the camera seeing the box's border (texels outside the grid read the
    border density 0)."""
    core = core_dr
    if mode == "nee_ess":
        sp = fbm_scene(width=40, height=40, mode="nee", use_ess=True, interp=interp)
    else:
        sp = fbm_scene(width=40, height=40, mode=mode, interp=interp)
    setup_core(core, sp)
    core("vpt_set_option", b"schedule", float(sched))
    feats = (ctypes.c_int * 2)(3, 6)  # normal, depth
    out = []
    for tex in (0, 1):
        core("vpt_set_option", b"density_texture", float(tex))
        core("vpt_set_use_feature_maps", feats, 2)
        s, _ = gpu_render(core, sp, 3, stats=False)
        maps = []
        # normal (3 channels) and mean depth (channel 0 only: channel 1, the depth's standard deviation,
        # is a square root of a difference of float sums that float atomics add in any order)
        for fid, ch in ((3, 3), (6, 1)):
            m = np.zeros(ch * sp.width * sp.height, np.float32)
            core("vpt_get_feature_map", fid, m.ctypes.data_as(ctypes.c_void_p), ch, 0, None)
            maps.append(m)
        core("vpt_set_use_feature_maps", feats, 0)
        s2, _ = gpu_render(core, sp, 3, stats=False)  # without features: the refill kernel
        out.append((s, maps, s2))
    core("vpt_set_option", b"density_texture", 1.0)
    core("vpt_set_option", b"schedule", 2.0)
    (a, ma, a2), (b, mb, b2) = out
    assert np.allclose(a, b, rtol=1e-12, atol=1e-12)
    assert np.allclose(a2, b2, rtol=1e-12, atol=1e-12)
    for x, y in zip(ma, mb):
        # float atomics add the frames' values in any order; normals can cancel to ~0
        assert np.allclose(x, y, rtol=1e-5, atol=1e-5 * float(np.abs(x).max()))


@pytest.mark.parametrize("build", ["default", "dr"])
def test_environment_map_level0_matches_reference_shader(core, core_dr, build):
    """Level 0 of the core's importance pyramid against OctahedralMapper.glsl run on the CPU
    (tests/golden/image_filters.npz).  CUDA's atan2f / asinf differ from the C library's in the last ulp
    on some arguments, which moves a bilinear lookup by that much, and a texel whose largest of 25
    sub-samples changes hands moves by more: >= 99.9 % of the texels within rtol 1e-5, all within 1e-3
    (the parity build, with double-rounded transcendentals: >= 99.99 %); the oracle, on the C library,
    matches the shader bit for bit."""
    from tests.harness import image_golden

    core = core if build == "default" else core_dr
    octa, _ = image_golden()
    for key, (env, ref) in sorted(octa.items()):
        res = ref.shape[0]
        levels = int(np.log2(res))
        total = sum((1 << (levels - l)) ** 2 for l in range(levels))
        d = torch.from_numpy(np.ascontiguousarray(env)).cuda()
        out = torch.empty(total, device="cuda")
        assert core.lib.vpt_build_environment_pyramid(dptr(d), env.shape[1], env.shape[0], levels, dptr(out), None) == 0
        torch.cuda.synchronize()
        got = out.cpu().numpy()[:res * res].reshape(res, res)
        close = np.isclose(got, ref, rtol=1e-5, atol=1e-6)
        rel = float(np.max(np.abs(got - ref) / np.maximum(np.abs(ref), 1e-6)))
        print(f"[{build}] {key}: within 1e-5 {close.mean():.6f}, max relative difference {rel:.3g}")
        assert close.mean() >= (0.999 if build == "default" else 0.9999), key
        assert rel < 1e-3, key


def test_eaw_compute_path_matches_reference_shader(core):
    """The core's EAW with the compute path's colour weight (ref_compute_quirk) against the compute stage
    of EAWDenoise.glsl run on the CPU (tests/golden/image_filters.npz); tolerance as in the CPU pin."""
    from tests.harness import image_golden

    _, eaw = image_golden()
    for key, (color, pos, nrm, it, phi, ref) in sorted(eaw.items()):
        h, w = color.shape[:2]
        dc, dp, dn = (torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (color, pos, nrm))
        out = torch.empty_like(dc)
        assert core.lib.vpt_eaw_denoise_rgba(dptr(dc), dptr(dp), dptr(dn), w, h, it, phi[0], phi[1], phi[2], 1,
                                             dptr(out), None) == 0
        torch.cuda.synchronize()
        assert np.allclose(out.cpu().numpy(), ref, rtol=1e-5, atol=2e-5), key
