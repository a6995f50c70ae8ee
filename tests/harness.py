"""Test harness: drives the CUDA core through its C ABI and sets up the same scene in the CPU oracle.

The oracle side recomputes everything from the raw grid with its own code (bounds, normalisation,
supervoxels, occupancy, environment pyramid); only the camera matrix is taken from the core so that
both sides start every path from the same float matrix.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from cloudrendering_b200 import _lib
from cloudrendering_b200._lib import check, farr
from oracle import bridge

MODE = {"delta": 0, "spectral_delta": 1, "ratio": 2, "decomposition": 3, "rrt": 4, "nee": 5, "spectral_nee": 6,
        "rrt_unbiased": 9}
INTERP = {"nearest": 0, "stochastic": 1, "trilinear": 2}
ENV = {"default": 0, "black": 1, "single": 2, "constant_sun": 3, "image": 4}


def cloud_block(xs, ys, zs, value=1.0, empty_boundary=False):
    """createCloudBlock (test/VolumetricPathTracingTestData.cpp:32-61)."""
    g = np.full((zs, ys, xs), value, np.float32)
    if empty_boundary and xs >= 3 and ys >= 3 and zs >= 3:
        g[:] = 0.0
        g[1:zs - 1, 1:ys - 1, 1:xs - 1] = value
    return g


def supervoxel_size(nx, ny, nz, s=8):
    """SuperVoxelGrid constructors (SuperVoxelGrid.cpp:46-58)."""
    if nx < s or ny < s or nz < s:
        while not (nx % s == 0 and ny % s == 0 and nz % s == 0):
            s //= 2
    return s


class Core:
    """One VptContext."""

    def __init__(self, device=0, variant="default"):
        self.lib = _lib.load(variant)
        c = ctypes.c_void_p()
        st = self.lib.vpt_create(ctypes.byref(c), device)
        if st != 0:
            raise RuntimeError(f"vpt_create failed: {st}")
        self.ctx = c.value

    def __call__(self, name, *args):
        check(getattr(self.lib, name)(self.ctx, *args), name, self.ctx, self.lib)

    def close(self):
        if self.ctx:
            self.lib.vpt_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        self.close()


class SceneSpec:
    def __init__(self, grid=None, mode="delta", interp="stochastic", extinction=1024.0, albedo=0.9, g=0.5,
                 width=64, height=64, seed_offset=0, max_bounces=0, env="default", linear_rgb=0,
                 sun_dir=(0.5826, 0.7660, 0.2717), sun_intensity=(2.6, 2.6 * 0.961538462, 2.6 * 0.884615385),
                 sky_color=(1.0, 1.0, 1.0), cam_pos=(0.0, 0.0, 0.8), cam_target=(0.0, 0.0, 0.0),
                 fovy=2.0 * math.atan(0.5), near=0.01, far=100.0, max_grid_extent=0.25, env_rgba=None,
                 use_ess=False, env_intensity=(1.0, 1.0, 1.0), ess_ref_compat=False, lights=None,
                 extinction_base=(1.0, 1.0, 1.0), albedo_rgb=None, sdt_prob=2, emission=None, emission_cap=1.0,
                 emission_strength=1.0, tf=None, iso=False, iso_value=0.5, iso_color=(0.4, 0.4, 0.4), env_rot=None,
                 tf_albedo_strength=0.0, iso_brdf="Lambertian", brdf_params=None, iso_type="Density",
                 clip_plane=None, close_iso=False):
        self.__dict__.update(locals())
        del self.__dict__["self"]


LIGHT_TYPES = ["Point Light", "Spotlight", "Directional Light"]
ISO_BRDFS = {"Lambertian": 0, "Blinn Phong": 1, "Ambient": 2, "Cook Torrance": 3, "Disney (2012)": 4}
# setBrdfParameter keys in slot order, with the pass's defaults (VolumetricPathTracingPass.hpp:410-419)
BRDF_KEYS = ["subsurface", "metallic", "specular", "specular_tint", "roughness", "anisotropic", "sheen",
             "sheen_tint", "clearcoat", "clearcoat_gloss"]
BRDF_DEFAULTS = [0.0, 0.0, 0.5, 0.0, 0.5, 0.0, 0.0, 0.5, 0.0, 1.0]


def gradient_magnitude(grid):
    """The gradient-magnitude field of gradient isosurfaces (VolumetricPathTracingPass.cpp:690-727) in
    float32: central differences between neighbours clamped to the grid over their index distance,
    sqrt(dx^2 + dy^2 + dz^2); grid [z, y, x]."""
    g = np.ascontiguousarray(grid, np.float32)

    def diff(axis):
        n = g.shape[axis]
        idx = np.arange(n)
        lo, hi = np.maximum(idx - 1, 0), np.minimum(idx + 1, n - 1)
        shape = [1, 1, 1]
        shape[axis] = n
        return (np.take(g, hi, axis=axis) - np.take(g, lo, axis=axis)) / (hi - lo).astype(np.float32).reshape(shape)

    dz, dy, dx = diff(0), diff(1), diff(2)
    return np.sqrt((dx * dx + dy * dy) + dz * dz).astype(np.float32)


def clip_values(sp):
    """The clip plane's normal as the pass uploads it (glm::normalize: v * inversesqrt(dot(v, v)), in
    float32) and its distance, or None."""
    if sp.clip_plane is None:
        return None
    v = np.array(sp.clip_plane[:3], np.float32)
    dd = np.float32(np.float32(v[0] * v[0]) + np.float32(v[1] * v[1])) + np.float32(v[2] * v[2])
    inv = np.float32(np.float32(1.0) / np.sqrt(np.float32(dd), dtype=np.float32))
    return [float(np.float32(c * inv)) for c in v] + [float(np.float32(sp.clip_plane[3]))]


def brdf_values(sp):
    """The ten BRDF parameters of a SceneSpec as float32 values."""
    vals = list(BRDF_DEFAULTS)
    for k, v in (sp.brdf_params or {}).items():
        vals[BRDF_KEYS.index(k)] = v
    return [float(np.float32(v)) for v in vals]
LIGHT_SPACES = ["World", "View", "View Orientation"]
LIGHT_DEFAULTS = dict(type="Point Light", space="View", spot_total_width=0.0981747704, spot_falloff_start=0.0245436926,
                      color=(1.0, 0.961538462, 0.884615385), intensity=0.5, position=(0.0, 0.0, 0.0), use_distance=1,
                      spot_direction=(0.0, 0.0, -1.0))


def _f32s(v):
    return repr(float(np.float32(v)))


def light_properties(light: dict):
    """(key, value) strings of vpt_set_light_property for a light dict (defaults of LightEditorWidget)."""
    L = dict(LIGHT_DEFAULTS)
    L.update(light)
    vec = lambda v: " ".join(_f32s(x) for x in v)  # noqa: E731
    return [("type", L["type"]), ("space", L["space"]), ("color", vec(L["color"])), ("intensity", _f32s(L["intensity"])),
            ("position", vec(L["position"])), ("use_distance", "1" if L["use_distance"] else "0"),
            ("spot_direction", vec(L["spot_direction"])), ("spot_total_width", _f32s(L["spot_total_width"])),
            ("spot_falloff_start", _f32s(L["spot_falloff_start"]))]


def light_floats(lights):
    """16 floats per light for the oracle and the reference driver."""
    out = np.zeros(256, np.float32)
    for i, light in enumerate(lights or []):
        L = dict(LIGHT_DEFAULTS)
        L.update(light)
        out[16 * i:16 * i + 15] = [LIGHT_TYPES.index(L["type"]), LIGHT_SPACES.index(L["space"]), L["spot_total_width"],
                                   L["spot_falloff_start"], *L["color"], L["intensity"], *L["position"],
                                   1.0 if L["use_distance"] else 0.0, *L["spot_direction"]]
    return [float(v) for v in out]


def setup_core(core: Core, sp: SceneSpec):
    core("vpt_set_max_grid_extent", sp.max_grid_extent)
    g = np.ascontiguousarray(sp.grid, np.float32)
    nz, ny, nx = g.shape
    core("vpt_set_dense_grid", g.ctypes.data_as(ctypes.c_void_p), nx, ny, nz, 0)
    core("vpt_set_vpt_mode", MODE[sp.mode])
    core("vpt_set_grid_interpolation", INTERP[sp.interp])
    core("vpt_set_extinction_scale", sp.extinction)
    core("vpt_set_extinction_base", farr(list(sp.extinction_base)))
    core("vpt_set_scattering_albedo", farr(list(sp.albedo_rgb) if sp.albedo_rgb is not None else [sp.albedo] * 3))
    core("vpt_set_option", b"sdt_collision_probability", float(sp.sdt_prob))
    core("vpt_set_phase_g", sp.g)
    core("vpt_set_seed_offset", sp.seed_offset)
    core("vpt_set_use_linear_rgb", sp.linear_rgb)
    core("vpt_set_max_bounces", sp.max_bounces)
    core("vpt_set_sun", farr(sp.sun_dir), farr(sp.sun_intensity))
    core("vpt_set_sky_color", farr(sp.sky_color))
    core("vpt_set_environment_map_intensity_rgb", farr(sp.env_intensity))
    if sp.env == "image":
        rgba = np.ascontiguousarray(sp.env_rgba, np.float32)
        core("vpt_load_environment_map_rgba", rgba.ctypes.data_as(ctypes.c_void_p), rgba.shape[1], rgba.shape[0], 1, 0)
    else:
        core("vpt_set_builtin_environment_map", ENV[sp.env])
    core("vpt_set_env_map_rotation", farr(list(sp.env_rot)) if sp.env_rot is not None else None)
    core("vpt_set_use_empty_space_skipping", 1 if sp.use_ess else 0)
    core("vpt_set_camera", farr(sp.cam_pos), farr(sp.cam_target), farr([0, 1, 0]), sp.fovy, sp.near, sp.far)
    core("vpt_clear_lights")
    core("vpt_set_use_lights", 1 if sp.lights else 0)
    for i, light in enumerate(sp.lights or []):
        core("vpt_add_light", None)
        for k, v in light_properties(light):
            core("vpt_set_light_property", i, k.encode(), v.encode())
    if sp.emission is not None:
        e = np.ascontiguousarray(sp.emission, np.float32)
        core("vpt_set_emission_grid", e.ctypes.data_as(ctypes.c_void_p), e.shape[2], e.shape[1], e.shape[0], 0)
        core("vpt_set_emission_cap", sp.emission_cap)
        core("vpt_set_emission_strength", sp.emission_strength)
    core("vpt_set_use_emission", 1 if sp.emission is not None else 0)
    core("vpt_set_emission_strength", sp.emission_strength)
    if sp.tf is not None:
        t = np.ascontiguousarray(sp.tf, np.float32)
        core("vpt_set_transfer_function", t.ctypes.data_as(ctypes.c_void_p), t.shape[0])
    core("vpt_set_use_transfer_function", 1 if sp.tf is not None else 0)
    core("vpt_set_tf_scattering_albedo_strength", float(sp.tf_albedo_strength))
    core("vpt_set_use_isosurfaces", 1 if sp.iso else 0)
    core("vpt_set_surface_brdf", sp.iso_brdf.encode())
    core("vpt_set_isosurface_type", sp.iso_type.encode())
    core("vpt_set_use_clip_plane", 1 if sp.clip_plane is not None else 0)
    core("vpt_set_close_isosurfaces", 1 if sp.close_iso else 0)
    if sp.clip_plane is not None:
        core("vpt_set_clip_plane_normal", *[float(c) for c in sp.clip_plane[:3]])
        core("vpt_set_clip_plane_distance", float(sp.clip_plane[3]))
    for k, v in zip(BRDF_KEYS, brdf_values(sp)):
        core("vpt_set_brdf_parameter", k.encode(), repr(v).encode())
    core("vpt_set_iso_value", sp.iso_value)
    core("vpt_set_iso_surface_color", *[float(c) for c in sp.iso_color])
    core("vpt_set_resolution", sp.width, sp.height)
    core("vpt_set_denoiser", 0)


def gpu_render(core: Core, sp: SceneSpec, frames: int, stats=True):
    """Renders `frames` frames from a reset film; returns (sum, sum_sq) as [H, W, 3] float64."""
    core("vpt_set_collect_statistics", 1 if stats else 0)
    core("vpt_reset_accumulation")
    core("vpt_render_frames", frames, None)
    core("vpt_synchronize", None)
    n = sp.width * sp.height * 3
    s = np.zeros(n, np.float64)
    sq = np.zeros(n, np.float64) if stats else None
    core("vpt_read_statistics", s.ctypes.data_as(ctypes.c_void_p),
         sq.ctypes.data_as(ctypes.c_void_p) if stats else None, 0, None)
    s = s.reshape(sp.height, sp.width, 3)
    if stats:
        sq = sq.reshape(sp.height, sp.width, 3)
    return s, sq


def _mat_mul(a, b):
    """Column-major 4x4 product in double, summation order of the core's mat_mul."""
    r = [0.0] * 16
    for c in range(4):
        for rr in range(4):
            acc = 0.0
            for k in range(4):
                acc += a[k * 4 + rr] * b[c * 4 + k]
            r[c * 4 + rr] = acc
    return r


def _mat_inverse(m):
    """Gauss-Jordan with partial pivoting, operation for operation as the core's mat_inverse."""
    a = [[m[c * 4 + r] for c in range(4)] + [1.0 if r == c else 0.0 for c in range(4)] for r in range(4)]
    for col in range(4):
        piv = col
        for r in range(col + 1, 4):
            if abs(a[r][col]) > abs(a[piv][col]):
                piv = r
        if piv != col:
            a[piv], a[col] = a[col], a[piv]
        inv = 1.0 / a[col][col]
        a[col] = [v * inv for v in a[col]]
        for r in range(4):
            if r == col:
                continue
            f = a[r][col]
            a[r] = [a[r][c] - f * a[col][c] for c in range(8)]
    return [a[r][4 + c] for c in range(4) for r in range(4)]


def _view_matrix(sp: SceneSpec):
    f32 = lambda v: float(np.float32(v))  # noqa: E731
    e = [f32(v) for v in sp.cam_pos]
    t = [f32(v) for v in sp.cam_target]
    up = [0.0, 1.0, 0.0]
    f = [t[i] - e[i] for i in range(3)]
    fl = math.sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2])
    f = [v / fl for v in f]
    s = [f[1] * up[2] - f[2] * up[1], f[2] * up[0] - f[0] * up[2], f[0] * up[1] - f[1] * up[0]]
    sl = math.sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2])
    s = [v / sl for v in s]
    u = [s[1] * f[2] - s[2] * f[1], s[2] * f[0] - s[0] * f[2], s[0] * f[1] - s[1] * f[0]]
    return [s[0], u[0], -f[0], 0.0, s[1], u[1], -f[1], 0.0, s[2], u[2], -f[2], 0.0,
            -(s[0] * e[0] + s[1] * e[1] + s[2] * e[2]), -(u[0] * e[0] + u[1] * e[1] + u[2] * e[2]),
            (f[0] * e[0] + f[1] * e[1] + f[2] * e[2]), 1.0]


def camera_inv_view(sp: SceneSpec):
    """inverse(view) as the core computes it for view-space lights (double, rounded to float)."""
    return [float(np.float32(v)) for v in _mat_inverse(_view_matrix(sp))]


def camera_inv_view_proj(sp: SceneSpec):
    """The core's camera (vpt_set_camera + compute_camera in vpt_context.cu) restated operation for
    operation in IEEE double from the float32-rounded inputs: look-at view, perspective with depth in
    [0, 1] and y flipped, Gauss-Jordan inverse, rounded to float.  Bit-identical to
    vpt_get_camera_matrices for the same SceneSpec."""
    f32 = lambda v: float(np.float32(v))  # noqa: E731
    view = _view_matrix(sp)
    aspect = float(sp.width) / float(sp.height) if sp.width > 0 and sp.height > 0 else 1.0
    th = math.tan(f32(sp.fovy) / 2.0)
    n, fa = f32(sp.near), f32(sp.far)
    proj = [0.0] * 16
    proj[0] = 1.0 / (aspect * th)
    proj[5] = -1.0 / th
    proj[10] = fa / (n - fa)
    proj[11] = -1.0
    proj[14] = -(fa * n) / (fa - n)
    inv = _mat_inverse(_mat_mul(proj, view))
    return [f32(v) for v in inv]


def camera_view_proj(sp: SceneSpec):
    """proj * view of the core's camera for `sp` (double, rounded to float; vpt_get_camera_matrices)."""
    f32 = lambda v: float(np.float32(v))  # noqa: E731
    view = _view_matrix(sp)
    aspect = float(sp.width) / float(sp.height) if sp.width > 0 and sp.height > 0 else 1.0
    th = math.tan(f32(sp.fovy) / 2.0)
    n, fa = f32(sp.near), f32(sp.far)
    proj = [0.0] * 16
    proj[0] = 1.0 / (aspect * th)
    proj[5] = -1.0 / th
    proj[10] = fa / (n - fa)
    proj[11] = -1.0
    proj[14] = -(fa * n) / (fa - n)
    return [f32(v) for v in _mat_mul(proj, view)]


def oracle_scene(core, sp: SceneSpec, frames: int, frame_count: int = 0) -> bridge.Scene:
    if core is not None:
        inv = (ctypes.c_float * 16)()
        vp = (ctypes.c_float * 16)()
        core("vpt_get_camera_matrices", inv, vp)
    else:
        inv = camera_inv_view_proj(sp)
    g = np.ascontiguousarray(sp.grid, np.float32)
    nz, ny, nx = g.shape
    vmin, vmax = bridge.minmax(g)
    dens = bridge.normalize(g, vmin, vmax)
    bmin, bmax = bridge.grid_bounds(nx, ny, nz, sp.max_grid_extent)
    f32 = np.float32
    vpu = [f32(n / (float(f32(b1)) - float(f32(b0)))) for n, b0, b1 in zip((nx, ny, nz), bmin, bmax)]
    border = (f32(0.0) - f32(vmin)) / (f32(vmax) - f32(vmin))
    sc = bridge.Scene(
        inv_view_proj=list(inv), width=sp.width, height=sp.height, frame_count=frame_count, num_frames=frames,
        seed_offset=sp.seed_offset, mode=MODE[sp.mode], interp=INTERP[sp.interp], max_bounces=sp.max_bounces,
        use_ess=1 if sp.use_ess else 0, box_min=bmin, box_max=bmax, nx=nx, ny=ny, nz=nz, vox_per_unit=vpu,
        border_density=float(border), extinction=float(f32(f32(sp.extinction_base[0]) * f32(sp.extinction))),
        albedo=float(f32(sp.albedo_rgb[0] if sp.albedo_rgb is not None else sp.albedo)),
        g=float(f32(sp.g)), env_kind=ENV[sp.env], use_linear_rgb=sp.linear_rgb, env_image_linear=1,
        sun_intensity=sp.sun_intensity, sky_color=sp.sky_color, env_intensity=sp.env_intensity, density=dens)
    sc.set("inv_view", camera_inv_view(sp))
    sc.set("num_lights", len(sp.lights or []))
    sc.set("env_is_black", 1 if sp.env == "black" else 0)
    sc.set("lights", light_floats(sp.lights))
    sc.set("ext_rgb", [float(f32(f32(b) * f32(sp.extinction))) for b in sp.extinction_base])
    sc.set("albedo_rgb", [float(f32(a)) for a in (sp.albedo_rgb if sp.albedo_rgb is not None else [sp.albedo] * 3)])
    sc.set("sdt_prob", int(sp.sdt_prob))
    if sp.emission is not None:  # the core's emission box and voxel scale (vpt_context.cu fill_params)
        e = np.ascontiguousarray(sp.emission, np.float32)
        enz, eny, enx = e.shape
        ebmin, ebmax = bridge.grid_bounds(enx, eny, enz, sp.max_grid_extent)
        sc.set("emission", e)
        sc.set("enx", enx)
        sc.set("eny", eny)
        sc.set("enz", enz)
        sc.set("emission_box_min", ebmin)
        sc.set("emission_vox_per_unit", [float(np.float32(n / (float(b1) - float(b0))))
                                         for n, b0, b1 in zip((enx, eny, enz), ebmin, ebmax)])
        sc.set("emission_cap", float(np.float32(sp.emission_cap)))
    sc.set("emission_strength", float(np.float32(sp.emission_strength)))
    if sp.tf is not None:
        t = np.ascontiguousarray(sp.tf, np.float32)
        sc.set("tf", t)
        sc.set("tf_size", t.shape[0])
    sc.set("tf_albedo_strength", float(np.float32(sp.tf_albedo_strength)))
    if sp.iso:
        sc.set("use_iso", 1)
        sc.set("iso_subdivisions", 2)
        sc.set("interp", 2)
        sc.set("iso_brdf", ISO_BRDFS[sp.iso_brdf])
        sc.set("brdf", brdf_values(sp))
        if sp.iso_type == "Gradient":
            vmin, vmax = bridge.minmax(g)
            sc.set("iso_grad", gradient_magnitude(g))
            sc.set("iso_norm_min", float(np.float32(vmin)))
            sc.set("iso_norm_range", float(np.float32(np.float32(vmax) - np.float32(vmin))))
    if sp.clip_plane is not None:
        sc.set("use_clip", 1)
        sc.set("clip", clip_values(sp))
        sc.set("iso_close", 1 if (sp.close_iso and sp.iso) else 0)
    sc.set("iso_value", float(np.float32(sp.iso_value)))
    sc.set("iso_color", [float(np.float32(c)) for c in sp.iso_color])
    if sp.env_rot is not None and sp.env == "image":
        sc.set("env_rot", 1)
        sc.set("env_rot_m", [float(np.float32(v)) for v in sp.env_rot])
    # sun direction normalised exactly like vpt_set_sun (float ops in order)
    d = np.array(sp.sun_dir, np.float32)
    dl = np.sqrt(np.float32(np.float32(d[0] * d[0]) + np.float32(d[1] * d[1])) + np.float32(d[2] * d[2]), dtype=np.float32)
    sc.set("sun_dir", [float(np.float32(d[i] / dl)) for i in range(3)])
    ext = f32(sp.extinction)
    if sp.mode == "rrt_unbiased":
        svs = supervoxel_size(nx, ny, nz)
        delta = [f32(b1) - f32(b0) for b0, b1 in zip(bmin, bmax)]
        svw = [(f32(svs) * dlt) / f32(n) for dlt, n in zip(delta, (nx, ny, nz))]
        for k, v in zip(("sv_size", "svx", "svy", "svz"), (svs, -(-nx // svs), -(-ny // svs), -(-nz // svs))):
            sc.set(k, v)
        sc.set("sv_world", [float(v) for v in svw])
        sc.set("sv_inv_world", [float(f32(1.0) / v) for v in svw])
        mn, mx, avg, _ = bridge.supervoxel_stats(dens, svs, 1)
        sc.set("sv_local", bridge.rrt_local(mn, mx, avg, float(ext), svs))
    elif sp.mode in ("decomposition", "rrt") or sp.use_ess:
        nee_like = sp.mode in ("nee", "spectral_nee")
        svs = 8 if sp.use_ess and nee_like else supervoxel_size(nx, ny, nz)
        svx, svy, svz = -(-nx // svs), -(-ny // svs), -(-nz // svs)
        delta = [f32(b1) - f32(b0) for b0, b1 in zip(bmin, bmax)]
        svw = [(f32(svs) * dlt) / f32(n) for dlt, n in zip(delta, (nx, ny, nz))]
        sc.set("sv_size", svs)
        sc.set("svx", svx)
        sc.set("svy", svy)
        sc.set("svz", svz)
        sc.set("sv_world", [float(v) for v in svw])
        halo = 0 if sp.interp == "nearest" else 1
        if nee_like:
            if sp.ess_ref_compat:  # the reference marks every block occupied (ComputeOccupancyGrid.glsl:108-109)
                sc.set("occupancy", np.ones(svx * svy * svz, np.uint8))
                sc.set("ess_ref_compat", 1)
            else:
                sc.set("occupancy", bridge.occupancy(dens, 8, halo, 0.0))
        else:
            mn, mx, avg, occ = bridge.supervoxel_stats(dens, svs, halo)
            if sp.mode == "rrt":
                sc.set("sv_data", bridge.rrt_params(mn, mx, avg, float(ext), svs))
            else:
                sc.set("sv_data", np.stack([mn, mx], axis=1).reshape(-1).copy())
    if sp.env == "image":
        rgba = np.ascontiguousarray(sp.env_rgba, np.float32)
        sc.set("env_rgba", rgba)
        sc.set("env_w", rgba.shape[1])
        sc.set("env_h", rgba.shape[0])
        sc.set("env_levels", 12)
        sc.set("env_pyramid", bridge.env_pyramid(rgba, 12))
    return sc


def path_agreement(a: np.ndarray, b: np.ndarray, rtol=1e-4, atol=1e-5) -> float:
    """Fraction of paths whose rgb radiance agrees within rtol/atol on every channel."""
    ok = np.all(np.abs(a - b) <= atol + rtol * np.abs(b), axis=-1)
    return float(ok.mean())


def z_scores(sum_a, sq_a, n_a, sum_b, sq_b, n_b):
    ma, mb = sum_a / n_a, sum_b / n_b
    va = np.maximum(sq_a / n_a - ma * ma, 0.0) * n_a / max(n_a - 1, 1)
    vb = np.maximum(sq_b / n_b - mb * mb, 0.0) * n_b / max(n_b - 1, 1)
    se = np.sqrt(va / n_a + vb / n_b)
    z = np.where(se > 0, (ma - mb) / np.where(se > 0, se, 1.0), np.where(np.abs(ma - mb) > 1e-7, np.inf, 0.0))
    return z


def binned_z(sum_a, sq_a, n_a, sum_b, sq_b, n_b, B=8):
    """Per-pixel radiance is heavy-tailed (rare paths that see the sun lobe: one such path among n
    samples moves a pixel's z by up to sqrt(n)), so agreement is judged on BxB-pixel bins (n*B*B
    samples per bin and side).  Returns (max |z| over the bins, fraction of pixels with |z| > 4)."""
    H, W = sum_a.shape[:2]
    h, w = H // B * B, W // B * B

    def binsum(x):
        return x[:h, :w].reshape(h // B, B, w // B, B, -1).sum(axis=(1, 3))

    zb = z_scores(binsum(sum_a), binsum(sq_a), n_a * B * B, binsum(sum_b), binsum(sq_b), n_b * B * B)
    zpix = z_scores(sum_a, sq_a, n_a, sum_b, sq_b, n_b)
    zb = np.abs(np.where(np.isfinite(zb), zb, 0.0))
    return float(zb.max()), float((np.abs(np.where(np.isfinite(zpix), zpix, 0.0)) > 4).mean())


def reference_scene(sp: SceneSpec, frames: int, frame_start: int = 0, inv=None):
    """The same scene for the reference's own shader code compiled for the CPU (oracle/_ref)."""
    from oracle import ref_bridge

    if inv is None:
        inv = camera_inv_view_proj(sp)
    g = np.ascontiguousarray(sp.grid, np.float32)
    nz, ny, nx = g.shape
    vmin, vmax = bridge.minmax(g)
    dens = bridge.normalize(g, vmin, vmax)
    bmin, bmax = bridge.grid_bounds(nx, ny, nz, sp.max_grid_extent)
    d = np.array(sp.sun_dir, np.float32)
    dl = np.sqrt(np.float32(np.float32(d[0] * d[0]) + np.float32(d[1] * d[1])) + np.float32(d[2] * d[2]),
                 dtype=np.float32)
    sc = ref_bridge.Scene(
        inv_view_proj=list(inv), width=sp.width, height=sp.height, frame_start=frame_start, num_frames=frames,
        seed_offset=sp.seed_offset, box_min=bmin, box_max=bmax, grid=g, nx=nx, ny=ny, nz=nz,
        linear_filter=1 if sp.interp == "trilinear" else 0, voxel_value_min=vmin, voxel_value_max=vmax,
        extinction=[float(np.float32(np.float32(b) * np.float32(sp.extinction))) for b in sp.extinction_base],
        albedo=list(sp.albedo_rgb) if sp.albedo_rgb is not None else [sp.albedo] * 3, g=sp.g,
        sun_dir=[float(np.float32(d[i] / dl)) for i in range(3)], sun_intensity=sp.sun_intensity,
        env_intensity=sp.env_intensity, is_env_black=1 if sp.env == "black" else 0, far_dist=sp.far,
        inv_view=camera_inv_view(sp), lights=light_floats(sp.lights))
    if sp.mode in ("decomposition", "rrt"):
        svs = supervoxel_size(nx, ny, nz)
        halo = 0 if sp.interp == "nearest" else 1
        mn, mx, avg, occ = bridge.supervoxel_stats(dens, svs, halo)
        data = bridge.rrt_params(mn, mx, avg, float(np.float32(sp.extinction)), svs) if sp.mode == "rrt" else \
            np.stack([mn, mx], axis=1).reshape(-1).copy()
        sc.set("sv_data", data)
        for k, v in zip(("svx", "svy", "svz", "sv_size"), (-(-nx // svs), -(-ny // svs), -(-nz // svs), svs)):
            sc.set(k, v)
    if sp.use_ess:
        # the reference's occupancy pass marks every block occupied (ComputeOccupancyGrid.glsl:108-109)
        sc.set("occupancy", np.ones((-(-nx // 8)) * (-(-ny // 8)) * (-(-nz // 8)), np.uint8))
        for k, v in zip(("ox", "oy", "oz", "occ_block"), (-(-nx // 8), -(-ny // 8), -(-nz // 8), 8)):
            sc.set(k, v)
    if sp.env == "image":
        rgba = np.ascontiguousarray(sp.env_rgba, np.float32)
        sc.set("env_rgba", rgba)
        sc.set("env_w", rgba.shape[1])
        sc.set("env_h", rgba.shape[0])
        sc.set("env_levels", 12)
        sc.set("env_pyramid", bridge.env_pyramid(rgba, 12))
    if sp.emission is not None:
        e = np.ascontiguousarray(sp.emission, np.float32)
        enz, eny, enx = e.shape
        ebmin, ebmax = bridge.grid_bounds(enx, eny, enz, sp.max_grid_extent)
        sc.set("emission", e)
        for k, v in (("enx", enx), ("eny", eny), ("enz", enz), ("emission_box_min", ebmin),
                     ("emission_box_max", ebmax), ("emission_cap", sp.emission_cap),
                     ("emission_strength", sp.emission_strength)):
            sc.set(k, v)
    sc.set("emission_strength", sp.emission_strength)
    if sp.tf is not None:
        t = np.ascontiguousarray(sp.tf, np.float32)
        sc.set("tf", t)
        sc.set("tf_size", t.shape[0])
    sc.set("tf_albedo_strength", float(np.float32(sp.tf_albedo_strength)))
    prob = ["max", "avg", "hist"][sp.sdt_prob]
    tracker = {"delta": "delta", "ratio": "ratio", "decomposition": "decomposition", "rrt": "rrt",
               "nee": "nee_ess" if sp.use_ess else "nee", "spectral_delta": f"sdt_{prob}",
               "spectral_nee": f"nees_{prob}"}[sp.mode]
    if sp.lights:
        tracker = f"nee_l{len(sp.lights)}"
    if sp.emission is not None:
        tracker += "_emission"
    if sp.tf is not None:
        tracker += "_tf_albedo" if sp.tf_albedo_strength > 0 else "_tf"
    sc.set("iso_value", sp.iso_value)
    sc.set("iso_color", sp.iso_color)
    if sp.iso:
        tracker += {"Lambertian": "_iso", "Blinn Phong": "_iso_blinn", "Ambient": "_iso_ambient",
                    "Cook Torrance": "_iso_cook", "Disney (2012)": "_iso_disney"}[sp.iso_brdf]
        sc.set("brdf", brdf_values(sp))
        if sp.iso_type == "Gradient":
            tracker = tracker.replace("_iso", "_isograd")
            sc.set("gradient", gradient_magnitude(g))
    if sp.env_rot is not None:
        sc.set("env_rot", [float(np.float32(v)) for v in sp.env_rot])
        tracker += "_rot"
    if sp.clip_plane is not None:
        sc.set("use_clip", 1)
        sc.set("clip", clip_values(sp))
        tracker += "_clip"
        if sp.close_iso and sp.iso:
            tracker += "_close"
    env = {"default": "default", "black": "black", "single": "single", "image": "image"}[sp.env]
    colour = "linear" if (sp.linear_rgb or env != "default") else "srgb"
    return sc, f"{tracker}__{sp.interp}__{env}__{colour}"


GOLDEN = __import__("os").path.join(__import__("os").path.dirname(__import__("os").path.abspath(__file__)),
                                    "golden", "ref_paths.npz")


def golden_cases():
    """Cases of tests/golden/ref_paths.npz (outputs of the reference's own shader code):
    name -> (SceneSpec, inv_view_proj, paths [H, W, 3], mean8 [H, W, 3])."""
    import json

    z = np.load(GOLDEN)
    meta = json.loads(str(z["meta"]))
    out = {}
    for name, m in meta.items():
        kw = {k: (tuple(v) if isinstance(v, list) else v) for k, v in m.items() if k not in ("variant", "grid")}
        kw["grid"] = z[m["grid"]]
        if name + "__env_rgba" in z:
            kw["env_rgba"] = z[name + "__env_rgba"]
        if name + "__emission" in z:
            kw["emission"] = z[name + "__emission"]
        if name + "__tf" in z:
            kw["tf"] = z[name + "__tf"]
        sp = SceneSpec(**kw)
        out[name] = (sp, list(z[name + "__inv_view_proj"]), z[name + "__paths"], z[name + "__mean8"])
    return out


# ---------------------------------------------------------------------------------------------
# Sparse (NanoVDB) grids

SPARSE_GOLDEN = __import__("os").path.join(__import__("os").path.dirname(__import__("os").path.abspath(__file__)),
                                           "golden", "sparse_grids.npz")
SPARSE_GRIDS = ["fbm24", "block8b", "block1", "ragged", "saturated40", "tiles256"]


def sparse_grid(name: str) -> np.ndarray:
    """Normalised dense grids [nz, ny, nx] of the sparse fixtures (as CloudData::getSparseDensityField
    reads them through getDataFloatAtNorm)."""
    if name == "fbm24":
        g = bridge.fbm(24, 2, base_frequency=3.0, contrast=3.5)
    elif name == "block8b":
        g = cloud_block(8, 8, 8, empty_boundary=True)
    elif name == "block1":
        g = cloud_block(1, 1, 1)
    elif name == "ragged":
        g = bridge.fbm((40, 24, 33), 7, base_frequency=3.0, contrast=3.5)
    elif name == "saturated40":
        # high contrast: many leaves whose 512 voxels are all 1.0 become active lower-node tiles
        g = bridge.fbm(40, 3, base_frequency=2.0, contrast=12.0)
    elif name == "tiles256":
        # a 128^3 constant region aligned to a lower node (pruned to an upper-node tile), a constant
        # 8^3 leaf (pruned to a lower-node tile) and an fBm block with ragged leaves
        g = np.zeros((256, 256, 256), np.float32)
        g[0:128, 0:128, 0:128] = 0.7
        g[0:8, 0:8, 136:144] = 0.5
        g[16:80, 160:224, 160:224] = bridge.fbm(64, 5, base_frequency=3.0, contrast=3.5)
    else:
        raise KeyError(name)
    vmin, vmax = bridge.minmax(g)
    return bridge.normalize(g, vmin, vmax)


def sparse_golden():
    """name -> dict(buf, ijk, value, dim, active, walks=[(origin, dir, lowest level, walk records)], meta)."""
    import json

    z = np.load(SPARSE_GOLDEN)
    meta = json.loads(str(z["meta"]))
    out = {}
    for name, m in meta.items():
        walks = []
        index, od = z[f"{name}__walk_index"], z[f"{name}__walk_od"]
        parts = {f: z[f"{name}__walk_{f}"] for f in ("voxel", "dim", "active", "level", "box", "t")}
        for (lv, start, n), ray in zip(index, od):
            walks.append((ray[:3], ray[3:], int(lv), {f: a[start:start + n] for f, a in parts.items()}))
        out[name] = dict(buf=z[f"{name}__buf"], ijk=z[f"{name}__ijk"], value=z[f"{name}__value"],
                         dim=z[f"{name}__dim"], active=z[f"{name}__active"], walks=walks, meta=m)
    return out


# ---------------------------------------------------------------------------------------------
# Supervoxel grids of the reference's own builders (tests/golden/make_supervoxel_golden.py)

SUPERVOXEL_GOLDEN = __import__("os").path.join(__import__("os").path.dirname(__import__("os").path.abspath(__file__)),
                                               "golden", "supervoxel_grids.npz")


def supervoxel_golden():
    """key -> dict(raw grid, interp, dims (gx, gy, gz, supervoxel size), extinction, minmax, occ_decomposition,
    rrt, occ_rrt) from SuperVoxelGrid.cpp compiled unmodified."""
    import json

    z = np.load(SUPERVOXEL_GOLDEN)
    meta = json.loads(str(z["meta"]))
    out = {}
    for key, m in meta.items():
        out[key] = dict(raw=z[m["grid"] + "__raw"], interp=m["interp"], dims=m["dims"], extinction=m["extinction"],
                        **{f: z[f"{key}__{f}"] for f in ("minmax", "occ_decomposition", "rrt", "occ_rrt")})
    return out


IMAGE_GOLDEN = __import__("os").path.join(__import__("os").path.dirname(__import__("os").path.abspath(__file__)),
                                          "golden", "image_filters.npz")


def image_golden():
    """(octahedral maps, EAW cases) of the reference's image shaders (tests/golden/make_image_golden.py):
    octa: name -> (env RGBA [h, w, 4], map [res, res]); eaw: key -> (color, position, normal, iterations,
    phi, output)."""
    import json

    z = np.load(IMAGE_GOLDEN)
    meta = json.loads(str(z["meta"]))
    octa, eaw = {}, {}
    for key, m in meta.items():
        if key.startswith("octa_"):
            octa[key] = (z[key + "__env"], z[key + "__map"])
        else:
            i = m["input"]
            eaw[key] = (z[i + "__color"], z[i + "__position"], z[i + "__normal"], m["iterations"], tuple(m["phi"]),
                        z[key + "__out"])
    return octa, eaw


SVGF_GOLDEN = __import__("os").path.join(__import__("os").path.dirname(__import__("os").path.abspath(__file__)),
                                         "golden", "svgf_frames.npz")


def svgf_golden():
    """(meta, inputs [frame] -> (noisy, normal, depth, fwidth, motion), outputs (iterations, frame) -> (out,
    colour history, moments history)) of the reference's SVGF shaders (tests/golden/make_svgf_golden.py)."""
    import json

    z = np.load(SVGF_GOLDEN)
    meta = json.loads(str(z["meta"]))
    inputs = [tuple(z[f"in{f}__{n}"] for n in ("noisy", "normal", "depth", "fwidth", "motion"))
              for f in range(meta["frames"])]
    outputs = {(it, f): (z[f"it{it}_f{f}__out"], z[f"it{it}_f{f}__color"], z[f"it{it}_f{f}__moments"])
               for it in meta["iterations"] for f in range(meta["frames"])}
    return meta, inputs, outputs


def svgf_close(got, exp):
    """Fraction of pixels whose every channel agrees to rtol 1e-4 (relative to |exp| + 1e-3)."""
    close = np.abs(got - exp) <= 1e-4 * (np.abs(exp) + 1e-3)
    return float(close.reshape(close.shape[0] * close.shape[1], -1).all(axis=1).mean())
