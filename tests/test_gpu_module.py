"""The drop-in module surface (initialize / render_frame / cleanup and the setters) on the GPU, with
the reference's error behaviour (Module.cpp:286-317)."""
import numpy as np
import pytest
import torch

from cloudrendering_b200 import vpt

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def module():
    vpt.initialize()
    yield
    vpt.cleanup()


def test_render_frame_cpu_and_cuda_shapes():
    for dev in ("cpu", "cuda"):
        for c in (3, 4):
            t = torch.zeros((c, 40, 56), dtype=torch.float32, device=dev)
            out = vpt.render_frame(t, 2)
            assert out.shape == (c, 40, 56) and out.dtype == torch.float32 and out.device == t.device
            assert torch.isfinite(out).all()
            if c == 4:
                assert torch.all(out[3] == 1.0)


def test_accumulation_continues_across_calls():
    vpt.set_vpt_mode_from_name("Delta Tracking")
    t = torch.zeros((3, 32, 32), dtype=torch.float32, device="cuda")
    vpt.set_seed_offset(0)  # resets accumulation
    a = vpt.render_frame(t, 4)
    b = vpt.render_frame(t, 4)  # mean over 8 frames
    vpt.set_seed_offset(0)
    c = vpt.render_frame(t, 8)
    assert torch.allclose(b, c, rtol=1e-5, atol=1e-6)
    assert not torch.equal(a, b)


def test_errors_match_reference():
    with pytest.raises(RuntimeError, match="sizes"):
        vpt.render_frame(torch.zeros((32, 32)), 1)
    with pytest.raises(RuntimeError, match="channels"):
        vpt.render_frame(torch.zeros((2, 32, 32)), 1)
    with pytest.raises(RuntimeError, match="32-bit float"):
        vpt.render_frame(torch.zeros((3, 32, 32), dtype=torch.float64), 1)
    with pytest.raises(RuntimeError):
        vpt.set_denoiser("OptiX Denoiser")


def test_settings_surface_and_fbm_scene():
    vpt.set_max_grid_extent(0.5)
    vpt.generate_fbm_cloud(64, seed=1)
    bb = vpt.get_render_bounding_box()
    assert np.allclose(bb, [-0.5, 0.5, -0.5, 0.5, -0.5, 0.5])
    vpt.set_extinction_scale(200.0)
    vpt.set_scattering_albedo([0.99, 0.99, 0.99])
    vpt.set_phase_g(0.85)
    vpt.set_use_builtin_environment_map("Constant Sky + Sun")
    vpt.set_sky_color([0.2, 0.2, 0.2])
    vpt.set_sun([0.3, 0.8, 0.5], [5.0, 5.0, 5.0])
    vpt.set_camera_position([0.0, 0.3, 2.0])
    vpt.set_camera_target([0.0, 0.0, 0.0])
    vpt.set_camera_fovy(60.0)
    vpt.set_max_bounces(64)
    t = torch.zeros((4, 64, 64), dtype=torch.float32, device="cuda")
    for name in vpt.VPT_MODE_NAMES[:7]:  # every tracker, the spectral ones included
        vpt.set_vpt_mode_from_name(name)
        img = vpt.render_frame(t, 4)
        assert torch.isfinite(img).all() and img[:3].mean() > 0.0
    st = vpt.get_stats()
    assert st["paths"] > 0 and st["density_lookups"] > 0


def test_feature_maps_and_eaw():
    vpt.set_vpt_mode_from_name("Next Event Tracking")
    vpt.set_use_feature_maps(["Result", "First X", "Normal", "Depth", "Albedo", "Transmittance"])
    t = torch.zeros((3, 48, 48), dtype=torch.float32, device="cuda")
    img = vpt.render_frame(t, 8)
    pos = vpt.get_feature_map_from_string(t, "First X")
    assert pos.shape == (4, 48, 48)
    hit = pos[3]
    assert 0.0 < float(hit.mean()) <= 1.0
    tr = vpt.get_feature_map_from_string(t, "Transmittance")
    assert torch.allclose(tr[0] + hit, torch.ones_like(hit), atol=1e-5)
    vpt.set_denoiser("Edge-Avoiding À-Trous Wavelet Transform")
    vpt.set_denoiser_property("iterations", "3")
    den = vpt.render_frame(t, 8)
    assert den.shape == img.shape and torch.isfinite(den).all()
    assert float(den.std()) <= float(img.std()) * 1.05
    vpt.set_denoiser("SVGF")
    s = vpt.render_frame(t, 1)
    assert torch.isfinite(s).all()
    vpt.set_denoiser("None")


def test_normal_len1_depth_far_and_background_maps():
    """Normal (Length 1): the Normal map's rgb scaled to length 1 where longer than 1e-5, alpha 1
    (NormalizeNormals.glsl); Depth Far: mean of (event ? depth : far distance) (Clouds.glsl:219-227);
    Background: mean of (event ? skybox of the camera ray : the path's radiance) (Clouds.glsl:162-170),
    which under a single-colour sky is that colour at every pixel (the radiance of a path without
    an event is the sky it escapes to)."""
    vpt.set_vpt_mode_from_name("Delta Tracking")
    vpt.set_use_builtin_environment_map("Single Color")
    vpt.set_sun([0.3, 0.8, 0.5], [0.7, 0.5, 0.25])
    t = torch.zeros((3, 48, 64), dtype=torch.float32, device="cuda")
    vpt.set_use_feature_maps(["Normal", "First X", "Depth"])
    vpt.render_frame(t, 2)
    with pytest.raises(RuntimeError, match="Background"):
        vpt.get_feature_map_from_string(t, "Background")
    vpt.set_use_feature_maps(["Normal", "Normal (Length 1)", "First X", "Depth", "Depth Far", "Background"])
    img = vpt.render_frame(t, 6)
    normal = vpt.get_feature_map_from_string(t, "Normal")
    n1 = vpt.get_feature_map_from_string(t, "Normal (Length 1)")
    assert n1.shape == (4, 48, 64) and torch.all(n1[3] == 1.0)
    length = normal[:3].norm(dim=0)
    long_ = length > 1e-5
    assert torch.allclose(n1[:3][:, long_], (normal[:3] / length)[:, long_], rtol=1e-5, atol=1e-6)
    assert torch.equal(n1[:3][:, ~long_], normal[:3][:, ~long_])
    hit = vpt.get_feature_map_from_string(t, "First X")[3]
    depth = vpt.get_feature_map_from_string(t, "Depth")[0]
    far = vpt.get_feature_map_from_string(t, "Depth Far")
    assert far.shape == (1, 48, 64)
    assert torch.allclose(far[0], depth + (1.0 - hit) * 80.0, rtol=1e-6, atol=1e-5)
    assert 0.0 < float(hit.mean()) < 1.0  # events and misses both present
    bg = vpt.get_feature_map_from_string(t, "Background")
    assert bg.shape == (4, 48, 64) and torch.all(bg[3] == 1.0)
    miss = hit == 0.0
    colour = img[:, miss].mean(dim=1)  # pixels without events render the sky colour itself
    assert torch.allclose(img[:, miss], colour[:, None], rtol=1e-6)
    assert torch.allclose(bg[:3], colour[:, None, None].expand(3, 48, 64), rtol=1e-5)
    vpt.set_use_feature_maps([])
    vpt.set_use_builtin_environment_map("Default")


def test_emission_grid_with_next_event_tracking():
    """set_emission_field / set_use_emission / set_emission_cap / set_emission_strength: under a black
    sky an absorbed NEE path ends with (t^2, t^4, t^8) * strength, t = clamp(value * cap, 0, 1); a
    constant field 0.5 with cap 2 gives t = 1, i.e. strength on every channel."""
    vpt.set_vpt_mode_from_name("Next Event Tracking")
    vpt.set_use_builtin_environment_map("Black")
    t = torch.zeros((3, 32, 32), dtype=torch.float32, device="cuda")
    vpt.set_use_emission(False)
    vpt.set_seed_offset(0)
    dark = vpt.render_frame(t, 4).clone()
    assert float(dark.abs().max()) == 0.0
    vpt.set_emission_field(torch.full((8, 8, 8), 0.5))
    vpt.set_emission_cap(2.0)
    vpt.set_emission_strength(3.0)
    vpt.set_use_emission(True)
    lit = vpt.render_frame(t, 4)
    assert float(lit.mean()) > 0.0
    assert torch.equal(lit[0], lit[1]) and torch.equal(lit[1], lit[2])
    frac = lit[0] / 3.0  # fraction of the pixel's paths that were absorbed
    assert torch.all(frac <= 1.0 + 1e-6) and torch.allclose(frac * 4, torch.round(frac * 4), atol=1e-5)
    vpt.set_use_emission(False)
    vpt.set_use_builtin_environment_map("Default")


def test_transfer_function_table():
    """set_transfer_function_table / set_use_transfer_function: every density lookup is the table's
    alpha, so a transparent table under a single-colour sky leaves every delta-tracked path
    escaping to that colour; load_transfer_function_file names the missing sgl loader."""
    vpt.set_vpt_mode_from_name("Delta Tracking")
    vpt.set_use_builtin_environment_map("Single Color")
    vpt.set_sun([0.3, 0.8, 0.5], [0.6, 0.4, 0.2])
    t = torch.zeros((3, 32, 32), dtype=torch.float32, device="cuda")
    vpt.set_use_transfer_function(False)
    vpt.set_seed_offset(0)
    cloud = vpt.render_frame(t, 2).clone()
    table = np.zeros((16, 4), np.float32)
    table[:, 0] = 1.0
    vpt.set_transfer_function_table(table)
    vpt.set_use_transfer_function(True)
    clear = vpt.render_frame(t, 2)
    colour = torch.tensor([0.6, 0.4, 0.2], device="cuda")[:, None, None].expand(3, 32, 32)
    assert torch.allclose(clear, colour, rtol=1e-6)
    assert not torch.allclose(cloud, colour, rtol=1e-3)
    with pytest.raises(RuntimeError, match="sgl"):
        vpt.load_transfer_function_file("any.xml")
    with pytest.raises(RuntimeError, match="N x 4"):
        vpt.set_transfer_function_table(np.zeros((4, 3)))
    vpt.set_use_transfer_function(False)
    vpt.set_use_builtin_environment_map("Default")


def _check_isosurfaces():
    """set_use_isosurfaces and its settings: an iso value above every density finds no surface, so
    the image equals the trilinear render without isosurfaces bit for bit; a surface inside the cloud
    changes it; the types, BRDFs and trackers that are not built raise."""
    vpt.set_vpt_mode_from_name("Delta Tracking")
    vpt.set_grid_interpolation("Trilinear")
    vpt.set_extinction_scale(100.0)  # paths well below the 1000-iteration cap of the isosurface loop
    t = torch.zeros((3, 32, 32), dtype=torch.float32, device="cuda")
    vpt.set_use_isosurfaces(False)
    vpt.set_seed_offset(0)
    plain = vpt.render_frame(t, 2).clone()
    vpt.set_isosurface_type("Density")
    vpt.set_surface_brdf("Lambertian")
    vpt.set_iso_surface_color([0.8, 0.5, 0.3])
    vpt.set_iso_value(2.0)
    vpt.set_use_isosurfaces(True)
    vpt.set_seed_offset(0)
    none_found = vpt.render_frame(t, 2).clone()
    assert torch.equal(none_found, plain)
    vpt.set_iso_value(0.3)
    vpt.set_seed_offset(0)
    surf = vpt.render_frame(t, 2).clone()
    assert torch.isfinite(surf).all()
    assert not torch.allclose(surf, plain, rtol=1e-3)
    vpt.set_isosurface_type("Gradient")  # the gradient-magnitude field is built on the first render
    vpt.set_iso_value(0.02)
    vpt.set_seed_offset(0)
    grad = vpt.render_frame(t, 1).clone()
    assert torch.isfinite(grad).all()
    vpt.set_isosurface_type("Density")
    vpt.set_iso_value(0.3)
    for brdf in ("Blinn Phong", "Disney (2012)", "Cook Torrance", "Ambient", "Lambertian"):
        vpt.set_surface_brdf(brdf)
        vpt.set_seed_offset(0)
        assert torch.isfinite(vpt.render_frame(t, 1)).all()
    vpt.set_brdf_parameter("roughness", "0.3")
    vpt.set_brdf_parameter("no_such_key", "1")  # ignored, as in the reference
    with pytest.raises(RuntimeError, match="number"):
        vpt.set_brdf_parameter("metallic", "abc")
    vpt.set_brdf_parameter("roughness", "0.5")
    with pytest.raises(RuntimeError):
        vpt.set_iso_surface_color([0.1, 0.2])
    vpt.set_vpt_mode_from_name("Next Event Tracking")  # surface next-event estimation (USE_ISOSURFACE_NEE)
    vpt.set_seed_offset(0)
    assert torch.isfinite(vpt.render_frame(t, 1)).all()
    vpt.set_vpt_mode_from_name("Ratio Tracking")
    with pytest.raises(RuntimeError, match="delta"):
        vpt.render_frame(t, 1)
    vpt.set_use_isosurfaces(False)
    vpt.set_iso_value(0.5)
    vpt.set_vpt_mode_from_name("Delta Tracking")
    vpt.set_grid_interpolation("Stochastic")


def test_isosurfaces():
    try:
        _check_isosurfaces()
    finally:  # the module's state outlives the test: leave the defaults behind even after a failure
        vpt.set_use_isosurfaces(False)
        vpt.set_isosurface_type("Density")
        vpt.set_surface_brdf("Lambertian")
        vpt.set_iso_value(0.5)
        vpt.set_vpt_mode_from_name("Delta Tracking")
        vpt.set_grid_interpolation("Stochastic")
        vpt.set_extinction_scale(1024.0)


def test_load_xyz_file_grid_and_bounds(tmp_path):
    """load_cloud_file with a .xyz file: the normalised x-fastest grid reaches the renderer and the
    render box follows the header's voxel sizes (CloudData::computeGridBounds: size * voxel size,
    scaled so that the largest side is 2 * max grid extent, centred)."""
    import ctypes
    import struct

    from cloudrendering_b200 import _lib
    from tests.test_xyz_cpu import reference_grid, write_xyz

    sizes, voxel = (6, 4, 5), (0.5, 1.0, 0.75)
    values = np.random.default_rng(3).random(int(np.prod(sizes))).astype(np.float32)
    path = str(tmp_path / "cloud.xyz")
    write_xyz(path, values, sizes, voxel=voxel)
    vpt.set_max_grid_extent(0.25)
    vpt.load_cloud_file(path)
    lib, ctx = _lib.load(), vpt.context_handle()
    nx, ny, nz = sizes
    got = np.empty((nz, ny, nx), np.float32)
    _lib.check(lib.vpt_get_dense_grid(ctx, got.ctypes.data_as(ctypes.c_void_p), 0), "grid", ctx, lib)
    assert np.array_equal(got, reference_grid(values, sizes))
    ext = [np.float32(n) * np.float32(v) for n, v in zip(sizes, voxel)]
    ms = max(ext)
    half = [float(e * np.float32(0.25) / ms) for e in ext]
    box = vpt.get_render_bounding_box()
    assert np.allclose(box, [-half[0], half[0], -half[1], half[1], -half[2], half[2]], rtol=1e-6, atol=0)
    out = vpt.render_frame(torch.zeros((3, 16, 16), device="cuda"), 1)
    assert torch.isfinite(out).all()
    vpt.set_max_grid_extent(0.5)


def _sparse_box(wmin, wmax, gmin, gmax, ext):
    """CloudData::computeSparseGridMetadata (CloudData.cpp:1336-1344) in float32."""
    f = np.float32
    wmin, wmax, gmin, gmax = (np.array(v, f) for v in (wmin, wmax, gmin, gmax))
    diff = gmax - gmin
    md = diff.max()
    L = diff / md
    A = f(2.0) * f(ext) / md
    B = f(ext) * L - gmax * A
    return A * wmin + B, A * wmax + B


def test_global_world_bounding_box_places_loaded_nanovdb_grids():
    from tests.harness import sparse_golden

    buf = bytes(sparse_golden()["fbm24"]["buf"])
    vpt.set_max_grid_extent(0.5)
    vpt.load_nanovdb_grid(buf)
    w = vpt.get_vdb_world_bounding_box()
    wmin, wmax = [w[0], w[2], w[4]], [w[1], w[3], w[5]]
    lo, hi = _sparse_box(wmin, wmax, wmin, wmax, 0.5)
    box = vpt.get_render_bounding_box()
    assert np.allclose(box, [lo[0], hi[0], lo[1], hi[1], lo[2], hi[2]], rtol=1e-6, atol=1e-7)
    # a global box twice the grid's size, offset: the grid occupies its part of the unit-extent box
    g = [wmin[0] - 3.0, wmax[0] + 21.0, wmin[1], wmax[1] + 24.0, wmin[2] - 24.0, wmax[2]]
    vpt.set_global_world_bounding_box(g)
    vpt.load_nanovdb_grid(buf)
    lo, hi = _sparse_box(wmin, wmax, [g[0], g[2], g[4]], [g[1], g[3], g[5]], 0.5)
    box = vpt.get_render_bounding_box()
    assert np.allclose(box, [lo[0], hi[0], lo[1], hi[1], lo[2], hi[2]], rtol=1e-6, atol=1e-7)
    out = vpt.render_frame(torch.zeros((3, 16, 16), device="cuda"), 1)
    assert torch.isfinite(out).all()
    from cloudrendering_b200 import _lib
    _lib.check(_lib.load().vpt_set_global_world_bounding_box(vpt.context_handle(), None, None), "clear")
    vpt.generate_fbm_cloud(32, seed=1)  # a dense grid again, then the dense path
    vpt.set_use_sparse_grid(False)


def test_feature_map_type_selects_the_returned_image():
    vpt.set_max_grid_extent(0.5)
    vpt.generate_fbm_cloud(32, seed=1)
    vpt.set_use_builtin_environment_map("Default")
    t = torch.zeros((4, 24, 32), device="cuda")
    vpt.set_feature_map_type(6)  # Depth: (mean, standard deviation), blitted into RGBA
    vpt.set_seed_offset(0)
    depth_img = vpt.render_frame(t, 3).clone()
    want = vpt.get_feature_map(t, 6)
    assert torch.equal(depth_img[:2], want[:2])
    assert torch.all(depth_img[2] == 0) and torch.all(depth_img[3] == 1)
    assert float(depth_img[0].max()) > 0.0
    vpt.set_feature_map_type(0)
    vpt.set_seed_offset(0)
    res = vpt.render_frame(t, 3)
    assert not torch.equal(res[:2], depth_img[:2])
    vpt.set_use_feature_maps([])


def test_torch_ops_render_frame_matches_module():
    vpt.set_vpt_mode_from_name("Delta Tracking")
    t = torch.zeros((3, 20, 20), device="cuda")
    torch.ops.vpt.set_seed_offset(5)
    a = torch.ops.vpt.render_frame(t, 2).clone()
    vpt.set_seed_offset(5)
    b = vpt.render_frame(t, 2)
    assert torch.equal(a, b)


def test_env_map_rotation_identity_and_camera():
    rgba = torch.rand((4, 32, 64), device="cpu") * 2.0
    rgba[3] = 1.0
    vpt.load_environment_map_from_tensor(rgba)
    vpt.set_vpt_mode_from_name("Next Event Tracking")
    t = torch.zeros((3, 24, 24), device="cuda")
    vpt.disable_env_map_rot()
    a = vpt.render_frame(t, 2).clone()
    vpt.set_env_map_rot_quaternion([0.0, 0.0, 0.0, 1.0])  # identity: the same paths bit for bit
    b = vpt.render_frame(t, 2).clone()
    assert torch.equal(a, b)
    vpt.set_env_map_rot_euler_angles([1.2, 0.3, -0.5])
    c = vpt.render_frame(t, 2).clone()
    assert not torch.equal(a, c) and torch.isfinite(c).all()
    vpt.set_env_map_rot_camera()
    d = vpt.render_frame(t, 2)
    assert torch.isfinite(d).all()
    vpt.disable_env_map_rot()
    vpt.set_use_builtin_environment_map("Default")
    vpt.set_vpt_mode_from_name("Delta Tracking")


def test_clip_plane():
    """set_use_clip_plane / set_clip_plane_normal / set_clip_plane_distance: a plane through the cloud
    changes the image, the trackers it is not built for raise, and the setters check their arguments
    (the clipped paths themselves are pinned by the golden cases *_clip)."""
    t = torch.zeros((3, 32, 32), dtype=torch.float32, device="cuda")
    try:
        vpt.set_vpt_mode_from_name("Delta Tracking")
        vpt.set_seed_offset(0)
        plain = vpt.render_frame(t, 2).clone()
        vpt.set_use_clip_plane(True)
        vpt.set_clip_plane_normal([0.3, 0.5, 0.8])
        vpt.set_clip_plane_distance(0.0)
        vpt.set_seed_offset(0)
        cut = vpt.render_frame(t, 2).clone()
        assert torch.isfinite(cut).all()
        assert not torch.allclose(cut, plain, rtol=1e-3)
        with pytest.raises(RuntimeError, match="size 3"):
            vpt.set_clip_plane_normal([1.0, 0.0])
        with pytest.raises(RuntimeError, match="non-zero"):
            vpt.set_clip_plane_normal([0.0, 0.0, 0.0])
        vpt.set_vpt_mode_from_name("Decomposition Tracking")
        with pytest.raises(RuntimeError, match="clip plane"):
            vpt.render_frame(t, 1)
    finally:
        vpt.set_use_clip_plane(False)
        vpt.set_clip_plane_normal([1.0, 0.0, 0.0])
        vpt.set_clip_plane_distance(0.0)
        vpt.set_vpt_mode_from_name("Delta Tracking")
