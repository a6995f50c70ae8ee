"""ctypes bridge to ``oracle/_ref/libref_vpt.so``: the reference's own tracer shader compiled for the
CPU (TEST INFRASTRUCTURE ONLY).  Used to pin the oracle restatement and as the CPU reference arm."""
from __future__ import annotations

import ctypes
import os
from ctypes import c_char_p, c_float, c_int, c_uint8, c_uint32, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libref_vpt.so")


class RefScene(ctypes.Structure):
    _fields_ = [
        ("inv_view_proj", c_float * 16), ("width", c_int), ("height", c_int),
        ("frame_start", c_uint32), ("num_frames", c_uint32), ("seed_offset", c_uint32),
        ("box_min", c_float * 3), ("box_max", c_float * 3),
        ("grid", c_void_p), ("nx", c_int), ("ny", c_int), ("nz", c_int), ("linear_filter", c_int),
        ("voxel_value_min", c_float), ("voxel_value_max", c_float),
        ("extinction", c_float * 3), ("albedo", c_float * 3), ("g", c_float),
        ("sun_dir", c_float * 3), ("sun_intensity", c_float * 3), ("env_intensity", c_float * 3),
        ("sv_data", c_void_p), ("svx", c_int), ("svy", c_int), ("svz", c_int), ("sv_size", c_int),
        ("occupancy", c_void_p), ("ox", c_int), ("oy", c_int), ("oz", c_int), ("occ_block", c_int),
        ("env_rgba", c_void_p), ("env_w", c_int), ("env_h", c_int),
        ("env_pyramid", c_void_p), ("env_levels", c_int), ("is_env_black", c_int), ("far_dist", c_float),
        ("inv_view", c_float * 16), ("lights", c_float * 256),
        ("emission", c_void_p), ("enx", c_int), ("eny", c_int), ("enz", c_int),
        ("emission_box_min", c_float * 3), ("emission_box_max", c_float * 3), ("emission_cap", c_float),
        ("emission_strength", c_float), ("tf", c_void_p), ("tf_size", c_int),
        ("iso_value", c_float), ("iso_color", c_float * 3), ("env_rot", c_float * 9), ("prev_view_proj", c_float * 16),
        ("tf_albedo_strength", c_float), ("brdf", c_float * 10), ("gradient", c_void_p),
        ("use_clip", c_int), ("clip", c_float * 4),
    ]


_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def load():
    global _lib
    if _lib is None:
        lib = ctypes.CDLL(LIB_PATH)
        lib.ref_variant_count.restype = c_int
        lib.ref_variant_name.restype = c_char_p
        lib.ref_variant_name.argtypes = [c_int]
        lib.ref_find_variant.restype = c_int
        lib.ref_find_variant.argtypes = [c_char_p]
        lib.ref_render.restype = c_int
        lib.ref_render.argtypes = [c_int, ctypes.POINTER(RefScene), c_void_p, c_int]
        lib.ref_read_depth_feature.restype = c_int
        lib.ref_read_depth_feature.argtypes = [c_int, c_void_p]
        lib.ref_read_last_frame_feature.restype = c_int
        lib.ref_read_last_frame_feature.argtypes = [c_int, c_void_p]
        _lib = lib
    return _lib


def variant_name(tracker: str, interp: str, env: str, linear: bool) -> str:
    colour = "linear" if linear or env != "default" else "srgb"
    return f"{tracker}__{interp}__{env}__{colour}"


class Scene:
    def __init__(self, **kw):
        self.s = RefScene()
        self._keep = {}
        for k, v in kw.items():
            self.set(k, v)

    def set(self, k, v):
        if k in ("grid", "sv_data", "occupancy", "env_rgba", "env_pyramid", "emission", "tf", "gradient"):
            arr = None if v is None else np.ascontiguousarray(v)
            self._keep[k] = arr
            setattr(self.s, k, None if arr is None else arr.ctypes.data_as(c_void_p).value)
        elif isinstance(v, (list, tuple, np.ndarray)):
            a = getattr(self.s, k)
            for i, x in enumerate(v):
                a[i] = float(x)
        else:
            setattr(self.s, k, v)

    def render(self, variant: str, threads: int = 0) -> np.ndarray:
        lib = load()
        idx = lib.ref_find_variant(variant.encode())
        if idx < 0:
            raise KeyError(variant)
        out = np.empty((self.s.height, self.s.width, 4), np.float32)
        st = lib.ref_render(idx, ctypes.byref(self.s), out.ctypes.data_as(c_void_p), threads)
        if st != 0:
            raise RuntimeError("ref_render failed")
        return out

    @staticmethod
    def last_frame_feature(which: int, height: int, width: int) -> np.ndarray:
        """The last render's firstW (0), flowImage (1), flowReverseImage (2), reprojUVImage (3), normalImage
        (4), depthNablaImage (5) or depthFwidthImage (6), H x W x 4."""
        out = np.empty((height, width, 4), np.float32)
        if load().ref_read_last_frame_feature(which, out.ctypes.data_as(c_void_p)) != 0:
            raise RuntimeError("ref_read_last_frame_feature failed")
        return out

    @staticmethod
    def depth_feature(which: int, height: int, width: int) -> np.ndarray:
        """The last render's depthBlendedImage (which 0) or depthNearestOpaqueImage (1), H x W x 4."""
        out = np.empty((height, width, 4), np.float32)
        if load().ref_read_depth_feature(which, out.ctypes.data_as(c_void_p)) != 0:
            raise RuntimeError("ref_read_depth_feature failed")
        return out
