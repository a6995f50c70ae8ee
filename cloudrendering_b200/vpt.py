"""Drop-in mirror of the reference's ``vpt`` PyTorch module for the path-tracing hot path.

Same function names, argument meanings and error behaviour as ``src/PyTorch/vpt.pyi`` /
``src/PyTorch/Module.cpp`` of chrismile/CloudRendering for the functions on the tracing path; every
call goes to the CUDA core through its C ABI (include/vpt_b200.h).  torch is used only for tensors
and the current CUDA stream.

Differences, all documented supersets:
* ``render_frame`` on CUDA returns a fresh tensor instead of a view of an internal buffer that the
  next call overwrites (Module.cpp:687-692).
* extra entry points: ``set_density_field`` (CloudData::setDensityField), ``generate_fbm_cloud``,
  ``set_grid_interpolation``, ``set_max_bounces``, ``set_sun``, ``set_sky_color``, ``get_stats``,
  ``set_use_sparse_grid`` (the C++ pass's setUseSparseGrid), ``set_sparse_grid_fp16``,
  ``load_nanovdb_grid``.
* the builtin environment map list gains "Constant Sky + Sun" (constant sky plus the reference's
  Phong sun lobe, visible to every tracker).
"""
from __future__ import annotations

import ctypes
import math
import os
import struct
from typing import List, Optional

import numpy as np
import torch

from . import _lib
from ._lib import check, farr

# RenderSettings.hpp:37-41
VPT_MODE_NAMES = [
    "Delta Tracking", "Delta Tracking (Spectral)", "Ratio Tracking", "Decomposition Tracking",
    "Residual Ratio Tracking", "Next Event Tracking", "Next Event Tracking (Spectral)", "Isosurfaces",
    "Ray Marching (Emission/Absorption)",
    # no reference counterpart: next-event estimation with residual-ratio-tracked shadow rays and
    # supervoxel-majorant free paths (the reference's residual ratio mode is a biased estimator)
    "Residual Ratio Tracking (Unbiased)",
]
# RenderSettings.hpp:56-58
GRID_INTERPOLATION_TYPE_NAMES = ["Nearest", "Stochastic", "Trilinear"]
# RenderSettings.hpp:123-125 (+ one addition)
BUILTIN_ENV_MAP_NAMES = ["Default", "Black", "Single Color", "Constant Sky + Sun"]
# Denoiser.hpp:63-79 (names of the denoisers built here)
DENOISER_NAMES = {"None": 0, "Edge-Avoiding À-Trous Wavelet Transform": 1, "SVGF": 2,
                  "PyTorch Denoiser Module": -1}
# VolumetricPathTracingPass.hpp:74-80 (+ the new 2D transmittance feature)
VPT_FEATURE_MAP_NAMES = [
    "Result", "First X", "First W", "Normal", "Normal (Length 1)", "Cloud Only", "Depth", "Depth Far",
    "Flow", "Flow Reverse", "Depth (nabla)", "Depth (fwidth)", "Density", "Background", "Reprojected UV",
    "Depth Blended", "Depth Nearest Opaque", "Albedo", "Transmittance Volume",
    "Primary Ray Absorption Moments", "Scatter Ray Absorption Moments",
]
FEATURE_TRANSMITTANCE = 32
_FEATURE_BY_NAME = {n: i for i, n in enumerate(VPT_FEATURE_MAP_NAMES)}
_FEATURE_BY_NAME["Transmittance"] = FEATURE_TRANSMITTANCE


class _State:
    ctx: Optional[int] = None
    refcount: int = 0
    device: int = 0
    cam_pos = [0.0, 0.0, 0.8]
    cam_target = [0.0, 0.0, 0.0]
    cam_up = [0.0, 1.0, 0.0]
    fovy = 2.0 * math.atan(0.5)
    near = 1.0 / 512.0
    far = 80.0
    view_override: Optional[List[float]] = None
    grid_size = (0, 0, 0)
    env_intensity = 1.0
    # "PyTorch Denoiser Module" (runs on the host side of the boundary, pytorch_denoiser.py)
    torch_denoiser_active = False
    torch_denoiser_path = ""
    torch_denoiser = None
    torch_denoiser_loaded = ""
    user_feature_maps: List[int] = []
    feature_map_type: int = 0  # set_feature_map_type: the map render_frame returns (0 = Result)


S = _State()


def _ctx():
    if S.ctx is None:
        raise RuntimeError("vpt is not initialized: call initialize() first")
    return S.ctx


def _c(name: str, *args):
    lib = _lib.load()
    check(getattr(lib, name)(_ctx(), *args), name, _ctx())


def _apply_camera():
    if S.view_override is not None:
        _c("vpt_set_view_matrix", farr(S.view_override))
    else:
        _c("vpt_set_camera", farr(S.cam_pos), farr(S.cam_target), farr(S.cam_up), S.fovy, S.near, S.far)


def _fog_sphere(radius=0.25, voxel_size=0.01, half_width=3.0):
    """Dense counterpart of nanovdb::createFogVolumeSphere (the reference's default scene,
    Module.cpp:792-796): 1 inside, a linear ramp over `half_width` voxels at the surface."""
    n = int(math.ceil(2.0 * (radius + half_width * voxel_size) / voxel_size))
    c = (np.arange(n, dtype=np.float64) + 0.5) * voxel_size - n * voxel_size / 2.0
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    sdf = np.sqrt(x * x + y * y + z * z) - radius
    fog = np.clip(-sdf / (half_width * voxel_size), 0.0, 1.0).astype(np.float32)
    return np.ascontiguousarray(fog)


# ---- life cycle (Module.cpp:732-813) ----
def initialize() -> None:
    if S.refcount == 0:
        lib = _lib.load()
        ctx = ctypes.c_void_p()
        dev = torch.cuda.current_device() if torch.cuda.is_available() else 0
        st = lib.vpt_create(ctypes.byref(ctx), dev)
        if st != 0:
            raise RuntimeError(f"vpt_create failed: {lib.vpt_status_string(st).decode()}")
        S.ctx = ctx.value
        S.device = dev
        fog = _fog_sphere()
        set_density_field(torch.from_numpy(fog))
        _c("vpt_set_vpt_mode", 0)
        _c("vpt_set_use_linear_rgb", 1)
        _apply_camera()
    S.refcount += 1


def cleanup() -> None:
    if S.refcount <= 0:
        return
    S.refcount -= 1
    if S.refcount == 0:
        _lib.load().vpt_destroy(S.ctx)
        S.ctx = None


# ---- volume data ----
def set_density_field(density: torch.Tensor) -> None:
    """CloudData::setDensityField for a [Z, Y, X] (x fastest) float32 tensor on any device."""
    if density.dim() != 3:
        raise RuntimeError("Error in set_density_field: expected a 3D tensor [Z, Y, X].")
    d = density.detach().to(torch.float32).contiguous()
    nz, ny, nx = d.shape
    on_dev = 1 if d.is_cuda else 0
    _c("vpt_set_dense_grid", ctypes.c_void_p(d.data_ptr()), nx, ny, nz, on_dev)
    if on_dev:
        torch.cuda.synchronize(d.device)
    S.grid_size = (nx, ny, nz)


def generate_fbm_cloud(size, seed: int = 1, octaves: int = 6, lacunarity: float = 2.0, gain: float = 0.5,
                       base_frequency: float = 3.0, threshold: float = 0.3) -> None:
    """Seeded fBm Perlin cloud generated on the GPU (no reference counterpart)."""
    nx, ny, nz = (size, size, size) if isinstance(size, int) else size
    _c("vpt_generate_fbm_grid", nx, ny, nz, seed, octaves, lacunarity, gain, base_frequency, threshold)
    S.grid_size = (nx, ny, nz)


_NANOVDB_MAGIC = b"NanoVDB0"


def _nanovdb_grid_from_file(buf: bytes) -> bytes:
    """First grid of an uncompressed NanoVDB file: the file header and the grid data both start
    with the magic number; the grid's byte size is GridData::mGridSize (offset 32)."""
    if not buf.startswith(_NANOVDB_MAGIC):
        raise RuntimeError("Error in CloudData::loadFromNvdbFile: not a NanoVDB file.")
    start = buf.find(_NANOVDB_MAGIC, 8)
    if start < 0:
        raise RuntimeError("Error in CloudData::loadFromNvdbFile: no uncompressed grid found (compressed "
                           "NanoVDB files are not supported).")
    size = struct.unpack_from("<Q", buf, start + 32)[0]
    if start + size > len(buf):
        raise RuntimeError("Error in CloudData::loadFromNvdbFile: truncated grid.")
    return buf[start:start + size]


def load_nanovdb_grid(grid: bytes) -> None:
    """A NanoVDB float grid buffer (CloudData::setNanoVdbGridHandle): it replaces the dense grid and
    is rendered through the sparse path."""
    arr = np.frombuffer(grid, dtype=np.uint8)
    _c("vpt_set_nanovdb_grid", arr.ctypes.data_as(ctypes.c_void_p), arr.nbytes, 0)
    info = _sparse_info()
    S.grid_size = tuple(int(info.root_max[i] - info.root_min[i] + 1) for i in range(3))


def load_cloud_file(filename: str) -> None:
    """Loads a dense .xyz grid (CloudData::loadFromXyzFile, CloudData.cpp:236-317) or an
    uncompressed .nvdb NanoVDB file (CloudData::loadFromNvdbFile, CloudData.cpp:1360-1365)."""
    if not os.path.exists(filename):
        raise RuntimeError(f"Error in CloudData::loadFromFile: The file \"{filename}\" does not exist.")
    if filename.endswith(".nvdb"):
        with open(filename, "rb") as f:
            load_nanovdb_grid(_nanovdb_grid_from_file(f.read()))
        return
    if not filename.endswith(".xyz"):
        raise RuntimeError(f"Error in CloudData::loadFromFile: unsupported file format \"{filename}\".")
    with open(filename, "rb") as f:
        vx, vy, vz = struct.unpack_from("<3d", f.read(36), 12)
    grid = _read_xyz(filename)
    _c("vpt_set_voxel_size", vx, vy, vz)
    set_density_field(torch.from_numpy(grid))


load_volume_file = load_cloud_file


def _read_xyz(filename: str) -> np.ndarray:
    """A .xyz grid (CloudData::loadFromXyzFile, CloudData.cpp:236-317): [nz][ny][nx] float32 with the
    file's min-max normalisation (minimum at most 0)."""
    with open(filename, "rb") as f:
        buf = f.read()
    xs, ys, zs = struct.unpack_from("<3I", buf, 0)
    n = xs * ys * zs
    data = np.frombuffer(buf, dtype="<f4", count=n, offset=36).astype(np.float32)
    grid = data.reshape(xs, ys, zs).transpose(2, 1, 0).copy()  # z-fastest file -> x-fastest
    lo = min(0.0, float(grid.min()))
    hi = float(grid.max())
    if hi - lo > 1e-6:
        grid = (grid - np.float32(lo)) / np.float32(hi - lo)
    return np.ascontiguousarray(grid, dtype=np.float32)


# ---- emission (Module.cpp:826-832, 154-156; VolumetricPathTracingPass.cpp:897-906) ----
def load_emission_file(filename: str) -> None:
    """Loads the emission grid from a dense .xyz file (a second CloudData, normalised like the
    density; its box follows the grid's dimensions and the max grid extent)."""
    if not os.path.exists(filename):
        raise RuntimeError(f"Error in CloudData::loadFromFile: The file \"{filename}\" does not exist.")
    if not filename.endswith(".xyz"):
        raise RuntimeError(f"Error in CloudData::loadFromFile: unsupported emission file format \"{filename}\".")
    set_emission_field(torch.from_numpy(_read_xyz(filename)))


def set_emission_field(emission: torch.Tensor) -> None:
    """The emission grid as a [nz][ny][nx] float32 tensor (values scaled by the emission cap)."""
    if emission.dim() != 3:
        raise RuntimeError("Error in setEmissionField: expected a 3-D tensor.")
    e = emission.detach().to(torch.float32).contiguous()
    nz, ny, nx = e.shape
    on_dev = 1 if e.is_cuda else 0
    _c("vpt_set_emission_grid", ctypes.c_void_p(e.data_ptr()), int(nx), int(ny), int(nz), on_dev)


def set_use_emission(use_emission: bool) -> None:
    _c("vpt_set_use_emission", 1 if use_emission else 0)


def set_emission_cap(emission_cap: float) -> None:
    _c("vpt_set_emission_cap", float(emission_cap))


def set_emission_strength(emission_strength: float) -> None:
    _c("vpt_set_emission_strength", float(emission_strength))


# ---- transfer function (Module.cpp:106-112) ----
def set_use_transfer_function(_use_tf: bool) -> None:
    _c("vpt_set_use_transfer_function", 1 if _use_tf else 0)


def set_tf_scattering_albedo_strength(strength: float) -> None:
    """With a transfer function, spectral tracking scatters with mix(albedo, the table's rgb, strength)
    (Module.cpp:1352-1354; enabled for strength > 0)."""
    _c("vpt_set_tf_scattering_albedo_strength", float(strength))


def set_transfer_function_empty() -> None:
    """The empty transfer function of Module.cpp:1262-1276: opacity 0 and colour 0 over [0, 1]."""
    set_transfer_function_table(np.zeros((2, 4), np.float32))


def set_transfer_function_table(rgba) -> None:
    """The transfer-function texture as N x 4 RGBA values over the normalised density [0, 1] (the
    reference generates this table in sgl's TransferFunctionWindow)."""
    t = np.ascontiguousarray(np.asarray(rgba, dtype=np.float32))
    if t.ndim != 2 or t.shape[1] != 4 or t.shape[0] < 1:
        raise RuntimeError("Error in setTransferFunctionTable: expected an N x 4 RGBA table.")
    _c("vpt_set_transfer_function", t.ctypes.data_as(ctypes.c_void_p), int(t.shape[0]))


# ---- isosurfaces (Module.cpp:1163-1194) ----
def set_use_isosurfaces(_use_isosurfaces: bool) -> None:
    _c("vpt_set_use_isosurfaces", 1 if _use_isosurfaces else 0)


def set_iso_value(_iso_value: float) -> None:
    _c("vpt_set_iso_value", float(_iso_value))


def set_iso_surface_color(_iso_surface_color) -> None:
    _c("vpt_set_iso_surface_color", *_vec3(_iso_surface_color, "setIsoSurfaceColor"))


def set_isosurface_type(_isosurface_type: str) -> None:
    """"Density" or "Gradient" (isosurfaces of the gradient magnitude); unknown names are ignored."""
    _c("vpt_set_isosurface_type", str(_isosurface_type).encode())


def set_surface_brdf(_surface_brdf: str) -> None:
    """"Lambertian", "Blinn Phong", "Disney (2012)", "Cook Torrance" or "Ambient"; unknown names are
    ignored."""
    _c("vpt_set_surface_brdf", str(_surface_brdf).encode())


def set_brdf_parameter(key: str, value: str) -> None:
    """One BRDF parameter (subsurface, metallic, specular, specular_tint, roughness, anisotropic, sheen,
    sheen_tint, clearcoat, clearcoat_gloss) from its decimal string; unknown keys are ignored
    (src/PyTorch/Module.cpp:1196-1199)."""
    _c("vpt_set_brdf_parameter", str(key).encode(), str(value).encode())


def set_use_clip_plane(_use_clip_plane: bool) -> None:
    """Cuts every ray to the positive side of the clip plane (src/PyTorch/Module.cpp:1218-1220)."""
    _c("vpt_set_use_clip_plane", 1 if _use_clip_plane else 0)


def set_clip_plane_normal(_clip_plane_normal) -> None:
    """The clip plane's normal, three numbers (normalised by the renderer; Module.cpp:1222-1227)."""
    _c("vpt_set_clip_plane_normal", *_vec3(_clip_plane_normal, "setClipPlaneNormal"))


def set_clip_plane_distance(_clip_plane_distance: float) -> None:
    """The clip plane's distance along its normal (Module.cpp:1229-1231)."""
    _c("vpt_set_clip_plane_distance", float(_clip_plane_distance))


def set_close_isosurfaces(_close_isosurfaces: bool) -> None:
    """With isosurfaces and the clip plane on, the box faces and the clip plane close the isosurfaces
    (CLOSE_ISOSURFACES; src/PyTorch/Module.cpp:1209-1211)."""
    _c("vpt_set_close_isosurfaces", 1 if _close_isosurfaces else 0)


def set_num_isosurface_subdivisions(subdivisions: int) -> None:
    _c("vpt_set_num_isosurface_subdivisions", int(subdivisions))


def load_transfer_function_file(tf_file_path: str) -> None:
    raise RuntimeError("Error in loadTransferFunctionFile: transfer-function files are parsed by sgl's "
                       "TransferFunctionWindow, which this module does not include; pass the table to "
                       "set_transfer_function_table.")


def load_transfer_function_file_gradient(tf_file_path: str) -> None:
    raise RuntimeError("Error in loadTransferFunctionFileGradient: the gradient-magnitude transfer function "
                       "(gradient isosurfaces) is not built in this module.")


def set_transfer_function_range(_min_val: float, _max_val: float) -> None:
    raise RuntimeError("Error in setTransferFunctionRange: the range mapping is sgl's TransferFunctionWindow's, "
                       "which this module does not include; resample the table over the range and pass it to "
                       "set_transfer_function_table.")


def set_transfer_function_range_gradient(_min_val: float, _max_val: float) -> None:
    raise RuntimeError("Error in setTransferFunctionRangeGradient: the gradient-magnitude transfer function "
                       "(gradient isosurfaces) is not built in this module.")


def set_transfer_function_empty_gradient() -> None:
    raise RuntimeError("Error in setTransferFunctionEmptyGradient: the gradient-magnitude transfer function "
                       "(gradient isosurfaces) is not built in this module.")


def set_max_grid_extent(max_grid_extent: float) -> None:
    _c("vpt_set_max_grid_extent", float(max_grid_extent))


def set_global_world_bounding_box(global_bb_vec: List[float]) -> None:
    """Places NanoVDB grids loaded afterwards by this world box [xmin, xmax, ymin, ymax, zmin, zmax]
    instead of their own (Module.cpp:1383-1388; CloudData::computeSparseGridMetadata)."""
    if len(global_bb_vec) != 6:
        raise RuntimeError("Error in set_global_world_bounding_box: Expected vector of size 6.")
    b = [float(v) for v in global_bb_vec]
    _c("vpt_set_global_world_bounding_box", farr([b[0], b[2], b[4]]), farr([b[1], b[3], b[5]]))


def get_render_bounding_box() -> List[float]:
    out = (ctypes.c_float * 6)()
    _c("vpt_get_render_bounding_box", out)
    return [out[0], out[3], out[1], out[4], out[2], out[5]]


# ---- lights (Module.cpp:1088-1160, LightEditorWidget.cpp:89-103, 286-430) ----
LIGHT_TYPE_NAMES = ["Point Light", "Spotlight", "Directional Light"]
LIGHT_SPACE_NAMES = ["World", "View", "View Orientation"]


def set_use_lights(_use_lights: bool) -> None:
    _c("vpt_set_use_lights", 1 if _use_lights else 0)


def clear_lights() -> None:
    _c("vpt_clear_lights")


def add_light() -> None:
    _c("vpt_add_light", None)


def remove_light(light_idx: int) -> None:
    _c("vpt_remove_light", int(light_idx))


def set_light_property(light_idx: int, key: str, value: str) -> None:
    _c("vpt_set_light_property", int(light_idx), key.encode(), str(value).encode())


def load_lights_from_file(file_path: str) -> None:
    """The light editor's JSON format: {"lights": [{"type", "color": {r,g,b}, "intensity", "use_distance",
    "position": {x,y,z}, "space", "spot_total_width", "spot_falloff_start", "spot_direction": {x,y,z}}]}."""
    import json

    with open(file_path) as f:
        root = json.load(f)
    clear_lights()
    for i, node in enumerate(root.get("lights", [])):
        add_light()
        if "type" in node:
            set_light_property(i, "type", node["type"])
        if "color" in node:
            c = node["color"]
            set_light_property(i, "color", f"{c['r']!r} {c['g']!r} {c['b']!r}")
        if "intensity" in node:
            set_light_property(i, "intensity", repr(float(node["intensity"])))
        if "use_distance" in node:
            set_light_property(i, "use_distance", "1" if node["use_distance"] else "0")
        if "position" in node:
            p = node["position"]
            set_light_property(i, "position", f"{p['x']!r} {p['y']!r} {p['z']!r}")
        if "space" in node:
            set_light_property(i, "space", node["space"])
        for k in ("spot_total_width", "spot_falloff_start"):
            if k in node:
                set_light_property(i, k, repr(float(node[k])))
        if "spot_direction" in node:
            d = node["spot_direction"]
            set_light_property(i, "spot_direction", f"{d['x']!r} {d['y']!r} {d['z']!r}")


def set_use_headlight(_use_headlight: bool) -> None:
    """One view-space point light at the camera (Module.cpp:1131-1141)."""
    set_use_lights(_use_headlight)
    if _use_headlight:
        clear_lights()
        add_light()
        set_light_property(0, "space", "View")
        set_light_property(0, "position", "0 0 0")
        set_light_property(0, "use_distance", "1")


def set_use_headlight_distance(_use_headlight_distance: bool) -> None:
    set_light_property(0, "use_distance", "1" if _use_headlight_distance else "0")


def set_headlight_color(_headlight_color: List[float]) -> None:
    c = _vec3(_headlight_color, "set_headlight_color")
    set_light_property(0, "color", f"{c[0]!r} {c[1]!r} {c[2]!r}")


def set_headlight_intensity(_headlight_intensity: float) -> None:
    set_light_property(0, "intensity", repr(float(_headlight_intensity)))


# ---- sparse grids (VolumetricPathTracingPass::setUseSparseGrid; Module.cpp:1390-1400) ----
def set_use_sparse_grid(use_sparse: bool) -> None:
    """Render through a NanoVDB-style sparse volume built from the dense grid (the C++ pass's
    setUseSparseGrid; not exposed by the reference's Python module)."""
    _c("vpt_set_use_sparse_grid", 1 if use_sparse else 0)


def set_sparse_grid_fp16(use_fp16: bool) -> None:
    """Store the leaf values of the next sparse volume as IEEE half (no reference counterpart)."""
    _c("vpt_set_option", b"sparse_fp16", 1.0 if use_fp16 else 0.0)


def _sparse_info():
    info = _lib.VptSparseInfo()
    _c("vpt_get_sparse_grid_info", ctypes.byref(info))
    return info


def get_vdb_world_bounding_box() -> List[float]:
    i = _sparse_info()
    return [i.world_min[0], i.world_max[0], i.world_min[1], i.world_max[1], i.world_min[2], i.world_max[2]]


def get_vdb_index_bounding_box() -> List[int]:
    i = _sparse_info()
    return [i.root_min[0], i.root_max[0], i.root_min[1], i.root_max[1], i.root_min[2], i.root_max[2]]


def get_vdb_voxel_size() -> List[float]:
    i = _sparse_info()
    return [i.voxel_size[0], i.voxel_size[1], i.voxel_size[2]]


def get_volume_voxel_size() -> List[int]:
    nx, ny, nz = S.grid_size
    return [nz, ny, nx]


# ---- medium ----
def set_scattering_albedo(albedo: List[float]) -> None:
    _c("vpt_set_scattering_albedo", farr(_vec3(albedo, "setScatteringAlbedo")))


def set_extinction_scale(extinction_scale: float) -> None:
    _c("vpt_set_extinction_scale", float(extinction_scale))


def set_extinction_base(extinction_base: List[float]) -> None:
    _c("vpt_set_extinction_base", farr(_vec3(extinction_base, "setExtinctionBase")))


def set_phase_g(phase_g: float) -> None:
    _c("vpt_set_phase_g", float(phase_g))


def _vec3(v, where):
    if len(v) != 3:
        raise RuntimeError(f"Error in parseVector3: Expected vector of size 3 ({where}).")
    return [float(x) for x in v]


# ---- mode and sampling ----
def set_vpt_mode(mode: int) -> None:
    _c("vpt_set_vpt_mode", int(mode))


def set_vpt_mode_from_name(mode_name: str) -> None:
    if mode_name in VPT_MODE_NAMES:
        set_vpt_mode(VPT_MODE_NAMES.index(mode_name))


# SPECTRAL_DELTA_TRACKING_COLLISION_PROBABILITY_NAMES (src/PathTracer/RenderSettings.hpp:64-69)
SDT_COLLISION_PROBABILITY_NAMES = ["Max-based", "Avg-based", "Path History Avg-based"]


def set_spectral_delta_tracking_collision_probability(name: str) -> None:
    """Collision probabilities of the spectral trackers (VolumetricPathTracingPass::sdtCollisionProbability,
    set in the reference's GUI; default "Path History Avg-based")."""
    if name not in SDT_COLLISION_PROBABILITY_NAMES:
        raise RuntimeError(f"Error: invalid spectral delta tracking collision probability \"{name}\".")
    _c("vpt_set_option", b"sdt_collision_probability", float(SDT_COLLISION_PROBABILITY_NAMES.index(name)))


def set_grid_interpolation(name: str) -> None:
    if name not in GRID_INTERPOLATION_TYPE_NAMES:
        raise RuntimeError(f"Unknown grid interpolation type \"{name}\".")
    _c("vpt_set_grid_interpolation", GRID_INTERPOLATION_TYPE_NAMES.index(name))


def set_seed_offset(offset: int) -> None:
    _c("vpt_set_seed_offset", int(offset) & 0xFFFFFFFF)


def set_max_bounces(max_bounces: int) -> None:
    _c("vpt_set_max_bounces", int(max_bounces))


def set_use_empty_space_skipping(use: bool) -> None:
    _c("vpt_set_use_empty_space_skipping", 1 if use else 0)


# ---- lighting ----
def set_use_builtin_environment_map(env_map_name: str) -> None:
    if env_map_name in BUILTIN_ENV_MAP_NAMES:
        _c("vpt_set_builtin_environment_map", BUILTIN_ENV_MAP_NAMES.index(env_map_name))


def set_environment_map_intensity(intensity_factor: float) -> None:
    S.env_intensity = float(intensity_factor)
    _c("vpt_set_environment_map_intensity_rgb", farr([intensity_factor] * 3))


def set_environment_map_intensity_rgb(intensity_factor: List[float]) -> None:
    _c("vpt_set_environment_map_intensity_rgb", farr(_vec3(intensity_factor, "setEnvironmentMapIntensityFactorRgb")))


def set_sun(direction: List[float], intensity_rgb: List[float]) -> None:
    _c("vpt_set_sun", farr(_vec3(direction, "setSun")), farr(_vec3(intensity_rgb, "setSun")))


def set_sky_color(rgb: List[float]) -> None:
    _c("vpt_set_sky_color", farr(_vec3(rgb, "setSkyColor")))


def load_environment_map_from_tensor(env_map_tensor: torch.Tensor) -> None:
    """loadEnvironmentMapFromTensor (Module.cpp:898-963): CPU tensor [C, H, W] (C = 3 or 4) of uint8
    (sRGB), float16 or float32 (linear RGB), equirectangular."""
    if env_map_tensor.device.type != "cpu":
        raise RuntimeError("Error in loadEnvironmentMapFromTensor: Expected tensor using CPU memory.")
    c, h, w = env_map_tensor.shape
    if c not in (3, 4):
        raise RuntimeError("Error in loadEnvironmentMapFromTensor: Number of channels must be 3 or 4.")
    t = env_map_tensor.permute(1, 2, 0).contiguous()
    if t.dtype == torch.uint8:
        rgb = t.to(torch.float32) / 255.0
        linear = 0
    elif t.dtype in (torch.float16, torch.float32):
        rgb = t.to(torch.float32)
        linear = 1
    else:
        raise RuntimeError("Error in loadEnvironmentMapFromTensor: Unsupported pixel format.")
    rgba = torch.ones((h, w, 4), dtype=torch.float32)
    rgba[..., : min(c, 4)] = rgb[..., : min(c, 4)]
    rgba = rgba.contiguous()
    _c("vpt_load_environment_map_rgba", ctypes.c_void_p(rgba.data_ptr()), w, h, linear, 0)


def load_environment_map(filename: str) -> None:
    """Loads an equirectangular environment map stored as .npy (H, W, 3|4) float32 linear RGB.
    (.exr/.png need OpenEXR/libpng, which this build does not bundle.)"""
    if not filename.endswith(".npy"):
        raise RuntimeError(f"Error in loadEnvironmentMapImage: unsupported file format \"{filename}\".")
    arr = np.load(filename).astype(np.float32)
    load_environment_map_from_tensor(torch.from_numpy(arr).permute(2, 0, 1).contiguous())


# ---- environment-map rotation (Module.cpp:96-101, 979-1014; VolumetricPathTracingPass.cpp:1218-1284;
# the matrices of RotationWidget::getMat3, src/Utils/RotationWidget.cpp:62-77) ----
def _rot_x(a):
    c, s_ = math.cos(a), math.sin(a)
    return np.array([[1.0, 0.0, 0.0], [0.0, c, -s_], [0.0, s_, c]])


def _rot_y(a):
    c, s_ = math.cos(a), math.sin(a)
    return np.array([[c, 0.0, s_], [0.0, 1.0, 0.0], [-s_, 0.0, c]])


def _rot_z(a):
    c, s_ = math.cos(a), math.sin(a)
    return np.array([[c, -s_, 0.0], [s_, c, 0.0], [0.0, 0.0, 1.0]])


def _quat_matrix(x, y, z, w):
    """Rotation matrix of the quaternion w + xi + yj + zk (glm::toMat3 of a unit quaternion)."""
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                     [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                     [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])


def _set_env_rotation(m) -> None:
    """m: 3x3 row-major rotation (envMapDirRot); passed column-major to the core."""
    cm = np.asarray(m, np.float64).T.reshape(-1)
    _c("vpt_set_env_map_rotation", farr([float(np.float32(v)) for v in cm]))


def disable_env_map_rot() -> None:
    _c("vpt_set_env_map_rotation", None)


def set_env_map_rot_camera() -> None:
    """The environment image rotates with the camera (envMapRot = the view matrix, every frame)."""
    _c("vpt_set_env_map_rotation_camera")


def set_env_map_rot_euler_angles(euler_angles_vec: List[float]) -> None:
    """glm::eulerAngleYXZ(x, y, z) (radians): rotation about y by x, then x by y, then z by z."""
    a, b, c = _vec3(euler_angles_vec, "set_env_map_rot_euler_angles")
    _set_env_rotation(_rot_y(a) @ _rot_x(b) @ _rot_z(c))


def set_env_map_rot_yaw_pitch_roll(yaw_pitch_roll_vec: List[float]) -> None:
    """glm::yawPitchRoll(yaw, pitch, roll) (radians), the same matrix as the YXZ Euler angles."""
    a, b, c = _vec3(yaw_pitch_roll_vec, "set_env_map_rot_yaw_pitch_roll")
    _set_env_rotation(_rot_y(a) @ _rot_x(b) @ _rot_z(c))


def set_env_map_rot_angle_axis(_axis_vec: List[float], _angle: float) -> None:
    """glm::toMat3(glm::angleAxis(angle, axis / |axis|)) (the axis is used as given when shorter than 1e-6)."""
    ax = np.array(_vec3(_axis_vec, "set_env_map_rot_angle_axis"), np.float64)
    n = float(np.linalg.norm(ax))
    if n > 1e-6:
        ax = ax / n
    h = 0.5 * float(_angle)
    sh = math.sin(h)
    _set_env_rotation(_quat_matrix(ax[0] * sh, ax[1] * sh, ax[2] * sh, math.cos(h)))


def set_env_map_rot_quaternion(_quaternion_vec: List[float]) -> None:
    """glm::toMat3 of the quaternion given as (x, y, z, w) (parseQuaternion, Module.cpp:858-868)."""
    if len(_quaternion_vec) != 4:
        raise RuntimeError("Error in parseQuaternion: Expected vector of size 4.")
    x, y, z, w = (float(v) for v in _quaternion_vec)
    _set_env_rotation(_quat_matrix(x, y, z, w))


# ---- camera (VolumetricPathTracingModuleRenderer.cpp:303-324, Module.cpp:1282-1328) ----
def get_camera_position() -> List[float]:
    return list(S.cam_pos)


def get_camera_fovy() -> float:
    return S.fovy


def get_camera_view_matrix() -> List[float]:
    inv = (ctypes.c_float * 16)()
    vp = (ctypes.c_float * 16)()
    _c("vpt_get_camera_matrices", inv, vp)
    if S.view_override is not None:
        return list(S.view_override)
    e = np.array(S.cam_pos, np.float64)
    f = np.array(S.cam_target, np.float64) - e
    f /= np.linalg.norm(f)
    s = np.cross(f, np.array(S.cam_up, np.float64))
    s /= np.linalg.norm(s)
    u = np.cross(s, f)
    m = [s[0], u[0], -f[0], 0.0, s[1], u[1], -f[1], 0.0, s[2], u[2], -f[2], 0.0,
         -s.dot(e), -u.dot(e), f.dot(e), 1.0]
    return [float(x) for x in m]


def set_camera_position(camera_position: List[float]) -> None:
    S.cam_pos = _vec3(camera_position, "setCameraPosition")
    S.view_override = None
    _apply_camera()


def set_camera_target(camera_target: List[float]) -> None:
    S.cam_target = _vec3(camera_target, "setCameraTarget")
    S.view_override = None
    _apply_camera()


def set_camera_fovy(fovy: float) -> None:
    """Degrees, like the reference (Module.cpp:1325-1328)."""
    S.fovy = float(fovy) * math.pi / 180.0
    _apply_camera()


def overwrite_camera_view_matrix(view_matrix_data: List[float]) -> None:
    if len(view_matrix_data) != 16:
        raise RuntimeError("Error in overwriteCameraViewMatrix: expected 16 values.")
    S.view_override = [float(x) for x in view_matrix_data]
    _apply_camera()


def set_view_projection_matrix_as_previous() -> None:
    """Stores the current camera's view-projection as the previous one (setViewProjectionMatrixAsPrevious,
    Module.cpp:1339-1341): the Flow, Flow Reverse and Reprojected UV maps reproject into it.  The SVGF
    history follows the previous render's camera by itself."""
    _c("vpt_set_previous_view_projection", None)


# ---- denoising ----
def set_denoiser(denoiser_name: str) -> None:
    if denoiser_name not in DENOISER_NAMES:
        raise RuntimeError(f"Error in setDenoiser: Invalid denoiser name \"{denoiser_name}\".")
    S.torch_denoiser_active = DENOISER_NAMES[denoiser_name] < 0
    _c("vpt_set_denoiser", max(0, DENOISER_NAMES[denoiser_name]))
    if S.torch_denoiser is not None:
        S.torch_denoiser.reset_previous_frame()
    _apply_feature_maps()


def set_pytorch_denoiser_model_file(denoiser_model_file_path: str) -> None:
    """Module.cpp:1070 setPyTorchDenoiserModelFile: the model used by "PyTorch Denoiser Module"
    (loaded at the next rendered frame)."""
    S.torch_denoiser_path = str(denoiser_model_file_path)
    _c("vpt_reset_accumulation")
    if S.torch_denoiser_active:
        _ensure_torch_denoiser()
        _apply_feature_maps()


def _ensure_torch_denoiser():
    if not S.torch_denoiser_path:
        raise RuntimeError("Error: the PyTorch denoiser has no model file (set_pytorch_denoiser_model_file).")
    if S.torch_denoiser is None or S.torch_denoiser_loaded != S.torch_denoiser_path:
        from .pytorch_denoiser import PyTorchDenoiser
        d = PyTorchDenoiser(torch.device("cuda", S.device))
        d.load_model_from_file(S.torch_denoiser_path)
        S.torch_denoiser, S.torch_denoiser_loaded = d, S.torch_denoiser_path
    return S.torch_denoiser


def _apply_feature_maps() -> None:
    ids = list(S.user_feature_maps)
    if S.feature_map_type != 0:
        ids.append(S.feature_map_type)
    if S.torch_denoiser_active and S.torch_denoiser is not None:
        ids += [_FEATURE_BY_NAME[n] for n in S.torch_denoiser.renderer_feature_maps()]
    ids = sorted(set(ids))
    arr = (ctypes.c_int * max(1, len(ids)))(*ids)
    _c("vpt_set_use_feature_maps", arr, len(ids))


def set_denoiser_property(key: str, value: str) -> None:
    _c("vpt_set_denoiser_property", key.encode(), str(value).encode())


# ---- feature maps ----
def set_feature_map_type(type: int) -> None:  # noqa: A002 (the reference's argument name)
    """The feature map that render_frame returns instead of the result (setFeatureMapType,
    Module.cpp:1078-1081; VolumetricPathTracingPass.cpp:2287-2400 blits it as the scene image).  The
    map is accumulated while it is selected; 0 (Result) restores the radiance output."""
    t = int(type)
    if t != 0 and t not in _FEATURE_CHANNELS:
        raise RuntimeError(f"Error in setFeatureMapType: feature map {t} is not supported.")
    S.feature_map_type = t
    _apply_feature_maps()


def set_use_feature_maps(feature_map_names: List[str]) -> None:
    S.user_feature_maps = [_FEATURE_BY_NAME[n] for n in feature_map_names if n in _FEATURE_BY_NAME]
    _apply_feature_maps()


_FEATURE_CHANNELS = {1: 4, 2: 4, 3: 4, 4: 4, 5: 4, 6: 2, 7: 1, 8: 2, 9: 2, 10: 2, 11: 1, 12: 2, 13: 4, 14: 2, 15: 4,
                     16: 4, 17: 4, FEATURE_TRANSMITTANCE: 1}


def get_feature_map(input_tensor: torch.Tensor, feature_map: int) -> torch.Tensor:
    if feature_map == 0:
        return _read(input_tensor, input_tensor.size(0), "vpt_read_result")
    if feature_map not in _FEATURE_CHANNELS:
        raise RuntimeError(f"Error in getFeatureMap: feature map {feature_map} is not supported.")
    return _read(input_tensor, _FEATURE_CHANNELS[feature_map], "vpt_get_feature_map", feature_map)


def get_feature_map_from_string(input_tensor: torch.Tensor, feature_map: str) -> torch.Tensor:
    if feature_map not in _FEATURE_BY_NAME:
        raise RuntimeError(f"Error in getFeatureMapFromString: unknown feature map \"{feature_map}\".")
    return get_feature_map(input_tensor, _FEATURE_BY_NAME[feature_map])


def read_denoiser_features(albedo: Optional[torch.Tensor] = None, normal: Optional[torch.Tensor] = None,
                           depth: Optional[torch.Tensor] = None, transmittance: Optional[torch.Tensor] = None) -> None:
    """Writes the feature planes a learned denoiser reads (albedo and normal: 3 x H x W; depth mean and
    transmittance: H x W; leading dimensions of size 1 allowed) into contiguous float32 CUDA tensors of
    the current image size, in one launch on the current stream; None skips a plane."""
    if getattr(S, "last_hw", None) is None:
        raise RuntimeError("Error in readDenoiserFeatures: nothing rendered.")
    h, w = S.last_hw
    ptrs = []
    for t, planes in ((albedo, 3), (normal, 3), (depth, 1), (transmittance, 1)):
        if t is None:
            ptrs.append(None)
            continue
        if not t.is_cuda or t.dtype != torch.float32 or not t.is_contiguous() or t.numel() != planes * h * w:
            raise RuntimeError("Error in readDenoiserFeatures: expected a contiguous float32 CUDA tensor of "
                               f"{planes} x {h} x {w} values.")
        ptrs.append(ctypes.c_void_p(t.data_ptr()))
    _c("vpt_get_denoiser_features", *ptrs, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))


# ---- rendering (Module.cpp:286-317) ----
def _validate(input_tensor: torch.Tensor):
    if input_tensor.dim() != 3:
        raise RuntimeError("Error in renderFrame: inputTensor.sizes().size() != 3.")
    if input_tensor.size(0) not in (3, 4):
        raise RuntimeError("Error in renderFrame: The number of image channels is not equal to 3 or 4.")
    if input_tensor.dtype != torch.float32:
        raise RuntimeError("Error in renderFrame: The only data type currently supported is 32-bit float.")
    if input_tensor.device.type not in ("cpu", "cuda"):
        raise RuntimeError("Unsupported PyTorch device type.")


def _stream_of(t: torch.Tensor):
    if t.is_cuda:
        return ctypes.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)
    return ctypes.c_void_p(0)


def _read(input_tensor: torch.Tensor, channels: int, fn: str, feature: Optional[int] = None) -> torch.Tensor:
    h, w = input_tensor.size(1), input_tensor.size(2)
    # a host result lands in page-locked memory (torch's caching host allocator): the device-to-host
    # copy then runs at link speed instead of through a pageable staging copy
    out = torch.empty((channels, h, w), dtype=torch.float32, device=input_tensor.device,
                      pin_memory=not input_tensor.is_cuda)
    on_dev = 1 if out.is_cuda else 0
    ptr = ctypes.c_void_p(out.data_ptr())
    if feature is None:
        _c(fn, ptr, channels, on_dev, _stream_of(input_tensor))
    else:
        _c(fn, feature, ptr, channels, on_dev, _stream_of(input_tensor))
    return out


def render_frame(input_tensor: torch.Tensor, frame_count: int) -> torch.Tensor:
    """Renders `frame_count` 1-spp frames into the running mean and returns it as [C, H, W]."""
    _validate(input_tensor)
    c, h, w = input_tensor.shape
    if S.torch_denoiser_active:
        den = _ensure_torch_denoiser()
        _apply_feature_maps()
    _c("vpt_set_resolution", int(w), int(h))
    S.last_hw = (int(h), int(w))
    _c("vpt_render_frames", int(frame_count), _stream_of(input_tensor))
    if S.feature_map_type != 0:
        # the map blitted into the C-channel scene image: missing colour channels 0, missing alpha 1
        fm = get_feature_map(input_tensor, S.feature_map_type)
        k = fm.size(0)
        if k == c:
            return fm
        out = torch.zeros((c, h, w), dtype=torch.float32, device=fm.device)
        out[:min(k, c)] = fm[:min(k, c)]
        if c == 4 and k < 4:
            out[3] = 1.0
        return out
    if not S.torch_denoiser_active:
        return _read(input_tensor, c, "vpt_read_result")
    probe = torch.empty((4, h, w), dtype=torch.float32, device=torch.device("cuda", S.device))
    color = _read(probe, 4, "vpt_read_result")
    out = den.denoise(color, lambda name: get_feature_map_from_string(probe, name))
    return out[:c].to(input_tensor.device).contiguous()


def set_frame_index(first_frame: int) -> None:
    """Clears the accumulation and makes `first_frame` the seed frame index every cleared film starts
    from (frame sharding across GPUs; no reference counterpart)."""
    _c("vpt_set_frame_index", int(first_frame) & 0xFFFFFFFF)


def set_feature_frame_limit(frames: int) -> None:
    """Feature maps accumulate over the first `frames` frames of an accumulation only (0: every frame,
    as the reference does); later frames are traced without the feature pass (no reference
    counterpart; clears the accumulation)."""
    _c("vpt_set_option", b"feature_frames", float(frames))


def set_collect_statistics(enabled: bool) -> None:
    """Accumulates the per-pixel sum of squared frame radiance beside the FP64 film (no reference
    counterpart; clears the accumulation when the state changes)."""
    _c("vpt_set_collect_statistics", 1 if enabled else 0)


def get_film_moments(width: int, height: int, frames: int):
    """Mean and mean square of the accumulated frames' radiance, [3, H, W] float32 on the GPU
    (statistics collection must be on)."""
    s = torch.empty((height, width, 3), dtype=torch.float64, device=torch.device("cuda", S.device))
    q = torch.empty_like(s)
    _c("vpt_read_statistics", ctypes.c_void_p(s.data_ptr()), ctypes.c_void_p(q.data_ptr()), 1,
       ctypes.c_void_p(torch.cuda.current_stream(s.device).cuda_stream))
    inv = 1.0 / float(frames)
    return ((s * inv).float().permute(2, 0, 1).contiguous(), (q * inv).float().permute(2, 0, 1).contiguous())


def get_film_sum(width: int, height: int) -> torch.Tensor:
    """The FP64 film: the sum of the radiance of every accumulated frame, [3, H, W] float64 on the host."""
    _c("vpt_set_resolution", int(width), int(height))
    out = np.zeros(width * height * 3, np.float64)
    _c("vpt_read_statistics", out.ctypes.data_as(ctypes.c_void_p), None, 0, None)
    return torch.from_numpy(out.reshape(height, width, 3).transpose(2, 0, 1).copy())


def get_stats() -> dict:
    st = _lib.VptStats()
    _c("vpt_get_stats", ctypes.byref(st))
    return {"paths": st.paths, "density_lookups": st.density_lookups, "frames": st.frames,
            "error_flags": st.error_flags}


def reset_stats() -> None:
    _c("vpt_reset_stats")


def context_handle() -> int:
    """Raw VptContext* of the module's renderer (for C-ABI level tooling)."""
    return _ctx()


# torch.ops.vpt.<name> (the reference's TORCH_LIBRARY(vpt) registrations, Module.cpp:186-280)
from . import torch_ops as _torch_ops  # noqa: E402

_torch_ops.register(__import__(__name__, fromlist=["_"]))
