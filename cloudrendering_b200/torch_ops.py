"""The module's functions as PyTorch operators ``torch.ops.vpt.<name>``, for TorchScript and other
callers of the operator registry (the reference registers them with ``TORCH_LIBRARY(vpt, m)``,
src/PyTorch/Module.cpp:186-280, next to the pybind11 module).

Each operator forwards to the function of the same name in ``cloudrendering_b200.vpt``; its schema is
derived from that function's annotations.  Registration happens once, when ``vpt`` is imported.
"""
from __future__ import annotations

import inspect

import torch

# names registered by the reference's TORCH_LIBRARY block that this module implements, in its order
OPS = [
    "initialize", "cleanup", "render_frame", "load_cloud_file", "load_volume_file", "load_emission_file",
    "load_environment_map", "load_environment_map_from_tensor", "set_use_builtin_environment_map",
    "set_environment_map_intensity", "set_environment_map_intensity_rgb", "disable_env_map_rot",
    "set_env_map_rot_camera", "set_env_map_rot_euler_angles", "set_env_map_rot_yaw_pitch_roll",
    "set_env_map_rot_angle_axis", "set_env_map_rot_quaternion", "set_scattering_albedo", "set_extinction_base",
    "set_extinction_scale", "set_vpt_mode", "set_vpt_mode_from_name", "set_denoiser", "set_denoiser_property",
    "set_pytorch_denoiser_model_file", "set_use_transfer_function", "load_transfer_function_file",
    "set_transfer_function_empty", "set_tf_scattering_albedo_strength",
    "get_camera_position", "get_camera_view_matrix", "get_camera_fovy", "set_camera_position", "set_camera_target",
    "overwrite_camera_view_matrix", "set_feature_map_type", "set_use_empty_space_skipping", "set_use_lights",
    "clear_lights", "add_light", "remove_light", "set_light_property", "load_lights_from_file", "set_use_headlight",
    "set_use_headlight_distance", "set_headlight_color", "set_headlight_intensity", "set_use_isosurfaces",
    "set_iso_value", "set_iso_surface_color", "set_isosurface_type", "set_surface_brdf", "set_brdf_parameter",
    "set_use_clip_plane", "set_clip_plane_normal", "set_clip_plane_distance", "set_close_isosurfaces",
    "set_num_isosurface_subdivisions", "set_seed_offset", "set_use_feature_maps", "get_feature_map",
    "get_feature_map_from_string", "set_phase_g", "set_view_projection_matrix_as_previous", "set_use_emission",
    "set_emission_strength", "set_emission_cap", "get_volume_voxel_size", "get_render_bounding_box",
    "set_max_grid_extent", "set_global_world_bounding_box", "get_vdb_world_bounding_box",
    "get_vdb_index_bounding_box", "get_vdb_voxel_size",
]

_TYPES = {"torch.Tensor": "Tensor", "List[float]": "float[]", "List[int]": "int[]", "List[str]": "str[]",
          "float": "float", "int": "int", "str": "str", "bool": "bool", "None": "()"}
# arguments without an annotation in the module (vectors of three floats)
_UNANNOTATED = "float[]"

_LIB = None


def schema(name: str, fn) -> str:
    sig = inspect.signature(fn)
    args = []
    for p in sig.parameters.values():
        ann = p.annotation
        t = _UNANNOTATED if ann is inspect.Parameter.empty else _TYPES[str(ann)]
        args.append(f"{t} {p.name}")
    ret = _TYPES[str(sig.return_annotation)]
    return f"{name}({', '.join(args)}) -> {ret}"


def register(module) -> None:
    """Defines torch.ops.vpt.<name> for every name of OPS (once per process)."""
    global _LIB
    if _LIB is not None:
        return
    lib = torch.library.Library("vpt", "DEF")
    for name in OPS:
        fn = getattr(module, name)
        lib.define(schema(name, fn))
        lib.impl(name, fn, "CompositeExplicitAutograd")
    _LIB = lib
