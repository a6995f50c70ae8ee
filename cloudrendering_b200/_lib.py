"""ctypes binding of ``libvpt_b200.so`` (the C ABI declared in include/vpt_b200.h).

The library is loaded from this package directory.  There is no fallback: if the shared library is
missing the import of the rendering entry points raises, naming the build command.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_float, c_int, c_uint32, c_uint64, c_void_p

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libvpt_b200.so")
LIB_PATH_DR = os.path.join(_HERE, "libvpt_b200_dr.so")


class VptStats(ctypes.Structure):
    _fields_ = [
        ("paths", c_uint64),
        ("density_lookups", c_uint64),
        ("frames", c_uint64),
        ("error_flags", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


VptCtxP = c_void_p
F3 = POINTER(c_float)

# name -> (restype, argtypes)
SIGNATURES = {
    "vpt_status_string": (c_char_p, [c_int]),
    "vpt_abi_version": (c_int, []),
    "vpt_kernel_launch_count": (c_uint64, []),
    "vpt_create": (c_int, [POINTER(c_void_p), c_int]),
    "vpt_destroy": (None, [VptCtxP]),
    "vpt_last_error": (c_char_p, [VptCtxP]),
    "vpt_set_dense_grid": (c_int, [VptCtxP, c_void_p, c_int, c_int, c_int, c_int]),
    "vpt_generate_fbm_grid": (c_int, [VptCtxP, c_int, c_int, c_int, c_uint32, c_int, c_float, c_float, c_float, c_float]),
    "vpt_get_dense_grid": (c_int, [VptCtxP, c_void_p, c_int]),
    "vpt_set_voxel_size": (c_int, [VptCtxP, c_double, c_double, c_double]),
    "vpt_set_max_grid_extent": (c_int, [VptCtxP, c_float]),
    "vpt_get_render_bounding_box": (c_int, [VptCtxP, F3]),
    "vpt_set_vpt_mode": (c_int, [VptCtxP, c_int]),
    "vpt_set_grid_interpolation": (c_int, [VptCtxP, c_int]),
    "vpt_set_extinction_scale": (c_int, [VptCtxP, c_float]),
    "vpt_set_extinction_base": (c_int, [VptCtxP, F3]),
    "vpt_set_scattering_albedo": (c_int, [VptCtxP, F3]),
    "vpt_set_phase_g": (c_int, [VptCtxP, c_float]),
    "vpt_set_seed_offset": (c_int, [VptCtxP, c_uint32]),
    "vpt_set_use_linear_rgb": (c_int, [VptCtxP, c_int]),
    "vpt_set_max_bounces": (c_int, [VptCtxP, c_int]),
    "vpt_set_builtin_environment_map": (c_int, [VptCtxP, c_int]),
    "vpt_set_environment_map_intensity_rgb": (c_int, [VptCtxP, F3]),
    "vpt_set_sun": (c_int, [VptCtxP, F3, F3]),
    "vpt_set_sky_color": (c_int, [VptCtxP, F3]),
    "vpt_load_environment_map_rgba": (c_int, [VptCtxP, c_void_p, c_int, c_int, c_int, c_int]),
    "vpt_set_camera": (c_int, [VptCtxP, F3, F3, F3, c_float, c_float, c_float]),
    "vpt_set_view_matrix": (c_int, [VptCtxP, F3]),
    "vpt_get_camera_matrices": (c_int, [VptCtxP, F3, F3]),
    "vpt_set_resolution": (c_int, [VptCtxP, c_int, c_int]),
    "vpt_reset_accumulation": (c_int, [VptCtxP]),
    "vpt_set_frame_index": (c_int, [VptCtxP, c_uint32]),
    "vpt_render_frames": (c_int, [VptCtxP, c_int, c_void_p]),
    "vpt_read_result": (c_int, [VptCtxP, c_void_p, c_int, c_int, c_void_p]),
    "vpt_render_frame": (c_int, [VptCtxP, c_int, c_void_p, c_int, c_int, c_void_p]),
    "vpt_set_collect_statistics": (c_int, [VptCtxP, c_int]),
    "vpt_read_statistics": (c_int, [VptCtxP, c_void_p, c_void_p, c_int, c_void_p]),
    "vpt_set_use_feature_maps": (c_int, [VptCtxP, POINTER(c_int), c_int]),
    "vpt_get_feature_map": (c_int, [VptCtxP, c_int, c_void_p, c_int, c_int, c_void_p]),
    "vpt_get_denoiser_features": (c_int, [VptCtxP, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "vpt_set_emission_grid": (c_int, [VptCtxP, c_void_p, c_int, c_int, c_int, c_int]),
    "vpt_set_use_emission": (c_int, [VptCtxP, c_int]),
    "vpt_set_emission_cap": (c_int, [VptCtxP, c_float]),
    "vpt_set_emission_strength": (c_int, [VptCtxP, c_float]),
    "vpt_set_transfer_function": (c_int, [VptCtxP, c_void_p, c_int]),
    "vpt_set_use_transfer_function": (c_int, [VptCtxP, c_int]),
    "vpt_set_tf_scattering_albedo_strength": (c_int, [VptCtxP, c_float]),
    "vpt_set_use_isosurfaces": (c_int, [VptCtxP, c_int]),
    "vpt_set_iso_value": (c_int, [VptCtxP, c_double]),
    "vpt_set_iso_surface_color": (c_int, [VptCtxP, c_double, c_double, c_double]),
    "vpt_set_isosurface_type": (c_int, [VptCtxP, c_char_p]),
    "vpt_set_surface_brdf": (c_int, [VptCtxP, c_char_p]),
    "vpt_set_brdf_parameter": (c_int, [VptCtxP, c_char_p, c_char_p]),
    "vpt_set_use_clip_plane": (c_int, [VptCtxP, c_int]),
    "vpt_set_clip_plane_normal": (c_int, [VptCtxP, c_double, c_double, c_double]),
    "vpt_set_clip_plane_distance": (c_int, [VptCtxP, c_double]),
    "vpt_set_close_isosurfaces": (c_int, [VptCtxP, c_int]),
    "vpt_set_num_isosurface_subdivisions": (c_int, [VptCtxP, c_int]),
    "vpt_get_stats": (c_int, [VptCtxP, POINTER(VptStats)]),
    "vpt_reset_stats": (c_int, [VptCtxP]),
    "vpt_synchronize": (c_int, [VptCtxP, c_void_p]),
    "vpt_set_use_empty_space_skipping": (c_int, [VptCtxP, c_int]),
    "vpt_set_option": (c_int, [VptCtxP, c_char_p, c_double]),
    "vpt_set_denoiser": (c_int, [VptCtxP, c_int]),
    "vpt_set_denoiser_property": (c_int, [VptCtxP, c_char_p, c_char_p]),
    "vpt_build_supervoxel_grid": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_int, c_void_p, c_void_p,
                                          c_void_p, c_void_p, c_void_p]),
    "vpt_build_rrt_params": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_float, c_int, c_void_p, c_void_p]),
    "vpt_set_env_map_rotation": (c_int, [c_void_p, c_void_p]),
    "vpt_set_previous_view_projection": (c_int, [c_void_p, c_void_p]),
    "vpt_set_env_map_rotation_camera": (c_int, [c_void_p]),
    "vpt_set_global_world_bounding_box": (c_int, [c_void_p, c_void_p, c_void_p]),
    "vpt_build_residual_ratio_grid": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_float, c_int, c_void_p, c_void_p]),
    "vpt_build_occupancy_grid": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_int, c_float, c_void_p,
                                         c_void_p]),
    "vpt_build_environment_pyramid": (c_int, [c_void_p, c_int, c_int, c_int, c_void_p, c_void_p]),
    "vpt_eaw_denoise_rgba": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int, c_int, c_float, c_float, c_float,
                                     c_int, c_void_p, c_void_p]),
    "vpt_batch_create": (c_int, [c_void_p, c_void_p, c_int]),
    "vpt_batch_destroy": (None, [c_void_p]),
    "vpt_batch_last_error": (c_char_p, [c_void_p]),
    "vpt_batch_set_option": (c_int, [c_void_p, c_char_p, c_double]),
    "vpt_batch_render": (c_int, [c_void_p, c_void_p, c_void_p]),
    "vpt_batch_autotune": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "vpt_batch_get_stats": (c_int, [c_void_p, c_void_p]),
    "vpt_batch_reset_stats": (c_int, [c_void_p]),
    "vpt_set_use_lights": (c_int, [c_void_p, c_int]),
    "vpt_clear_lights": (c_int, [c_void_p]),
    "vpt_add_light": (c_int, [c_void_p, c_void_p]),
    "vpt_remove_light": (c_int, [c_void_p, c_int]),
    "vpt_get_light_count": (c_int, [c_void_p, c_void_p]),
    "vpt_set_light_property": (c_int, [c_void_p, c_int, c_char_p, c_char_p]),
    "vpt_set_use_sparse_grid": (c_int, [c_void_p, c_int]),
    "vpt_set_nanovdb_grid": (c_int, [c_void_p, c_void_p, ctypes.c_size_t, c_int]),
    "vpt_get_sparse_grid_info": (c_int, [c_void_p, c_void_p]),
    "vpt_sparse_query": (c_int, [c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p]),
    "vpt_kpn_apply": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_int, c_int, c_int, c_int, c_int, c_void_p,
                              c_void_p]),
    "vpt_kpn_inv_iter": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_int, c_int, c_int, c_int,
                                 c_int, c_int, c_int, c_int, c_int, c_void_p, c_void_p]),
    "vpt_kpn_avg_pool2": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_void_p, c_void_p]),
    "vpt_kpn_reproject": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_int, c_int, c_int, c_void_p, c_void_p]),
    "vpt_eaw_denoise_rgba_noalloc": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int, c_int, c_float, c_float,
                                             c_float, c_int, c_void_p, c_void_p]),
    "vpt_gather_bench": (c_int, [c_void_p, ctypes.c_size_t, c_int, c_int, c_uint32, c_void_p, c_void_p]),
    "vpt_svgf_filter": (c_int, [c_void_p] * 9 + [c_int, c_int, c_float, c_float, c_int, c_void_p, c_void_p]),
    # learned denoiser network (csrc/vpt_unet.cu)
    "vpt_unet_conv3x3": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_int, c_int, c_int, c_int,
                                 c_int, c_int, c_void_p, c_void_p]),
    "vpt_unet_conv3x3_wgrad": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int, c_int, c_int, c_int, c_int,
                                       c_void_p, c_void_p]),
    "vpt_unet_wgrad_rows": (c_int, [c_int]),
    "vpt_unet_wgrad_splits": (c_int, [c_int, c_int, c_int, c_int, c_int, c_int]),
    "vpt_unet_set_conv_path": (c_int, [c_int]),
    "vpt_unet_set_conv_ksplit": (c_int, [c_int]),
    "vpt_unet_set_strip_kernel": (c_int, [c_int]),
    "vpt_unet_set_gather_stages": (c_int, [c_int]),
    "vpt_unet_rotate_weights": (c_int, [c_void_p, c_void_p, c_int, c_int, c_void_p]),
    "vpt_unet_pool2": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_int, c_void_p]),
    "vpt_unet_upcat": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int, c_int, c_int, c_int, c_void_p]),
    "vpt_unet_upcat_grad_lo": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int, c_int, c_int, c_int, c_void_p]),
    "vpt_unet_encoder_grad": (c_int, [c_void_p, c_int, c_int, c_void_p, c_void_p, c_void_p, c_int, c_int, c_int, c_int,
                                      c_void_p]),
    "vpt_unet_bias_grad": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_void_p]),
    "vpt_unet_reduce_grads": (c_int, [c_void_p, c_int, c_int, c_int, c_void_p, c_int, c_void_p, c_void_p, c_void_p]),
    "vpt_unet_adam": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, ctypes.c_long, c_float, c_float,
                              c_float, c_float, c_int, c_float, c_void_p]),
    "vpt_unet_to_bf16": (c_int, [c_void_p, c_void_p, ctypes.c_long, c_void_p]),
    "vpt_unet_pack_input": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                    c_int, c_int, c_int, c_void_p]),
    "vpt_unet_head_blocks": (c_int, [c_int, c_int, c_int]),
    "vpt_unet_kpn_combine": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int, c_void_p, c_int, c_int, c_int,
                                     c_void_p]),
    "vpt_unet_kpn_level_grad": (c_int, [c_void_p, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p,
                                        c_void_p, c_void_p, c_float, c_void_p, c_void_p, c_void_p, c_int, c_int, c_int,
                                        c_void_p]),
    "vpt_unet_add": (c_int, [c_void_p, c_void_p, c_void_p, ctypes.c_long, c_void_p]),
    "vpt_unet_kpn_head": (c_int, [c_void_p, c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int,
                                  c_int, c_int, c_float, c_void_p]),
}

class VptSparseInfo(ctypes.Structure):
    _fields_ = [("leaves", ctypes.c_uint64), ("tiles", ctypes.c_uint64), ("device_bytes", ctypes.c_uint64),
                ("table_origin", ctypes.c_int32 * 3), ("table_dim", ctypes.c_int32 * 3),
                ("root_min", ctypes.c_int32 * 3), ("root_max", ctypes.c_int32 * 3),
                ("box_min", c_float * 3), ("box_max", c_float * 3),
                ("world_min", ctypes.c_double * 3), ("world_max", ctypes.c_double * 3),
                ("voxel_size", ctypes.c_double * 3),
                ("fp16", ctypes.c_int32), ("lowest_level", ctypes.c_int32)]


_libs: dict = {}


def load(variant: str = "default") -> ctypes.CDLL:
    """Loads the library (once per variant) and installs the argument types.

    ``variant="dr"`` loads ``libvpt_b200_dr.so``: the same core with the tracer's transcendental
    functions evaluated in double precision and rounded once to float (used by the parity tests to
    compare paths one by one with the CPU oracle in the same mode)."""
    if variant in _libs:
        return _libs[variant]
    path = {"default": LIB_PATH, "dr": LIB_PATH_DR}[variant]
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build the CUDA core first (python -m cloudrendering_b200.build)")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _libs[variant] = lib
    return lib


def farr(values) -> ctypes.Array:
    vals = [float(v) for v in values]
    return (c_float * len(vals))(*vals)


class VptError(RuntimeError):
    """A call into the CUDA core returned a non-zero VptStatus."""

    def __init__(self, status: int, where: str, message: str):
        super().__init__(f"{where}: {message} (status {status})")
        self.status = status


def check(status: int, where: str, ctx=None, lib=None) -> None:
    if status == 0:
        return
    lib = lib or load()
    msg = lib.vpt_last_error(ctx).decode() if ctx else ""
    if not msg:
        msg = lib.vpt_status_string(status).decode()
    raise VptError(status, where, msg)
