"""ctypes bridge to the CPU oracle (TEST INFRASTRUCTURE ONLY).

Used by tests/, bench.py's cpu_baseline leg and __graft_entry__.smoke() as the checker.  The product
package never imports this module.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_float, c_int, c_uint8, c_uint32, c_uint64, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle_vpt.so")


class OracleScene(ctypes.Structure):
    _fields_ = [
        ("inv_view_proj", c_float * 16),
        ("width", c_int), ("height", c_int),
        ("frame_count", c_uint32), ("num_frames", c_uint32), ("seed_offset", c_uint32),
        ("mode", c_int), ("interp", c_int), ("max_bounces", c_int), ("use_ess", c_int), ("ess_ref_compat", c_int),
        ("box_min", c_float * 3), ("box_max", c_float * 3),
        ("nx", c_int), ("ny", c_int), ("nz", c_int),
        ("vox_per_unit", c_float * 3),
        ("border_density", c_float),
        ("extinction", c_float), ("albedo", c_float), ("g", c_float),
        ("sv_size", c_int), ("svx", c_int), ("svy", c_int), ("svz", c_int),
        ("sv_world", c_float * 3),
        ("env_kind", c_int), ("use_linear_rgb", c_int), ("env_image_linear", c_int),
        ("sun_dir", c_float * 3), ("sun_intensity", c_float * 3), ("sky_color", c_float * 3),
        ("env_intensity", c_float * 3),
        ("env_w", c_int), ("env_h", c_int), ("env_levels", c_int),
        ("density", c_void_p), ("sv_data", c_void_p), ("occupancy", c_void_p),
        ("env_rgba", c_void_p), ("env_pyramid", c_void_p),
        ("nanovdb", c_void_p), ("grid_min", c_float * 3), ("grid_max", c_float * 3),
        ("sparse_lowest_level", c_int), ("sparse_fp16", c_int),
        ("inv_view", c_float * 16), ("num_lights", c_int), ("env_is_black", c_int), ("lights", c_float * 256),
        ("ext_rgb", c_float * 3), ("albedo_rgb", c_float * 3), ("sdt_prob", c_int),
        ("emission", c_void_p), ("enx", c_int), ("eny", c_int), ("enz", c_int),
        ("emission_box_min", c_float * 3), ("emission_vox_per_unit", c_float * 3), ("emission_cap", c_float),
        ("emission_strength", c_float), ("tf", c_void_p), ("tf_size", c_int),
        ("use_iso", c_int), ("iso_value", c_float), ("iso_color", c_float * 3), ("iso_subdivisions", c_int),
        ("sv_inv_world", c_float * 3), ("sv_local", c_void_p),
        ("env_rot", c_int), ("env_rot_m", c_float * 9), ("tf_albedo_strength", c_float), ("iso_brdf", c_int),
        ("brdf", c_float * 10), ("iso_grad", c_void_p), ("iso_norm_min", c_float), ("iso_norm_range", c_float),
        ("use_clip", c_int), ("clip", c_float * 4), ("iso_close", c_int),
    ]


_lib = None


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            from . import build_oracle
            build_oracle.build()
        lib = ctypes.CDLL(LIB_PATH)
        P = POINTER
        lib.oracle_render.argtypes = [P(OracleScene), c_void_p, c_void_p, P(c_uint64), c_int]
        lib.oracle_render_rows.argtypes = [P(OracleScene), c_int, c_int, c_void_p, P(c_uint64), c_int]
        lib.oracle_trace_paths.argtypes = [P(OracleScene), c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_int]
        lib.oracle_fbm.argtypes = [c_void_p, c_int, c_int, c_int, c_uint32, c_int, c_float, c_float, c_float,
                                   c_float, c_float]
        lib.oracle_minmax.argtypes = [c_void_p, c_uint64, P(c_float), P(c_float)]
        lib.oracle_normalize.argtypes = [c_void_p, c_void_p, c_uint64, c_float, c_float]
        lib.oracle_grid_bounds.argtypes = [c_int, c_int, c_int, c_float, P(c_float), P(c_float)]
        lib.oracle_supervoxel_stats.argtypes = [c_void_p, c_int, c_int, c_int, c_int, c_int, c_void_p, c_void_p,
                                                c_void_p, c_void_p]
        lib.oracle_rrt_params.argtypes = [c_void_p, c_void_p, c_void_p, c_int, c_float, c_int, c_void_p]
        lib.oracle_rrt_local.argtypes = [c_void_p, c_void_p, c_void_p, c_int, c_float, c_int, c_void_p]
        lib.oracle_occupancy.argtypes = [c_void_p, c_int, c_int, c_int, c_int, c_int, c_float, c_void_p]
        lib.oracle_env_pyramid.argtypes = [c_void_p, c_int, c_int, c_int, c_void_p]
        lib.oracle_svgf_frame.argtypes = [c_void_p] * 9 + [c_int, c_int, c_float, c_float, c_int, c_void_p]
        lib.oracle_eaw.argtypes = [c_void_p, c_void_p, c_void_p, c_int, c_int, c_int, c_float, c_float, c_float,
                                   c_int, c_void_p]
        lib.oracle_rng_stream.argtypes = [c_uint32, c_int, c_void_p, c_void_p]
        lib.oracle_nanovdb_query.argtypes = [c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p]
        lib.oracle_nanovdb_hdda_walk.restype = c_int
        lib.oracle_nanovdb_hdda_walk.argtypes = [c_void_p, c_void_p, c_void_p, c_int, c_int, c_void_p, c_void_p,
                                                 c_void_p, c_void_p, c_void_p, c_void_p]
        lib.oracle_softmax_channels.argtypes = [c_void_p, c_int, c_int, c_int, c_int, c_void_p]
        lib.oracle_kpn_apply.argtypes = [c_void_p, c_void_p, c_int, c_int, c_int, c_int, c_int, c_int, c_int, c_void_p]
        lib.oracle_kpn_inv_iter_base.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_int, c_int,
                                                 c_int, c_int, c_int, c_int, c_int, c_int, c_int, c_void_p]
        lib.oracle_avg_pool2.argtypes = [c_void_p, c_int, c_int, c_int, c_void_p]
        lib.oracle_grid_sample.argtypes = [c_void_p, c_void_p, c_int, c_int, c_int, c_int, c_int, c_int, c_void_p]
        lib.oracle_set_double_rounded_math.argtypes = [c_int]
        lib.oracle_set_double_rounded_math.restype = None
        _lib = lib
    return _lib


def _ok(status: int) -> None:
    if status != 0:
        raise RuntimeError(f"oracle: scene rejected (status {status}): a tracker input is missing")


def _p(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(c_void_p)


def fbm(n, seed, octaves=6, lacunarity=2.0, gain=0.5, base_frequency=4.0, threshold=0.3, contrast=2.0):
    nx, ny, nz = (n, n, n) if isinstance(n, int) else n
    out = np.empty((nz, ny, nx), np.float32)
    load().oracle_fbm(_p(out), nx, ny, nz, seed, octaves, lacunarity, gain, base_frequency, threshold, contrast)
    return out


def minmax(v: np.ndarray):
    lo, hi = c_float(), c_float()
    load().oracle_minmax(_p(np.ascontiguousarray(v, np.float32)), v.size, ctypes.byref(lo), ctypes.byref(hi))
    return lo.value, hi.value


def normalize(v: np.ndarray, vmin: float, vmax: float) -> np.ndarray:
    v = np.ascontiguousarray(v, np.float32)
    out = np.empty_like(v)
    load().oracle_normalize(_p(v), _p(out), v.size, vmin, vmax)
    return out


def grid_bounds(nx, ny, nz, extent):
    bmin, bmax = (c_float * 3)(), (c_float * 3)()
    load().oracle_grid_bounds(nx, ny, nz, extent, bmin, bmax)
    return list(bmin), list(bmax)


def supervoxel_stats(dens: np.ndarray, sv: int, halo: int):
    nz, ny, nx = dens.shape
    gx, gy, gz = -(-nx // sv), -(-ny // sv), -(-nz // sv)
    mn = np.empty(gx * gy * gz, np.float32)
    mx = np.empty_like(mn)
    avg = np.empty_like(mn)
    occ = np.empty(gx * gy * gz, np.uint8)
    load().oracle_supervoxel_stats(_p(np.ascontiguousarray(dens, np.float32)), nx, ny, nz, sv, halo, _p(mn),
                                   _p(mx), _p(avg), _p(occ))
    return mn, mx, avg, occ


def rrt_params(mn, mx, avg, extinction, sv):
    out = np.empty(mn.size * 2, np.float32)
    load().oracle_rrt_params(_p(mn), _p(mx), _p(avg), mn.size, extinction, sv, _p(out))
    return out


def rrt_local(mn, mx, avg, extinction, sv):
    """Supervoxel grid of the unbiased residual ratio tracker: 4 floats per supervoxel."""
    out = np.empty(mn.size * 4, np.float32)
    load().oracle_rrt_local(_p(mn), _p(mx), _p(avg), mn.size, extinction, sv, _p(out))
    return out


def occupancy(dens, bs=8, halo=0, threshold=0.0):
    nz, ny, nx = dens.shape
    gx, gy, gz = -(-nx // bs), -(-ny // bs), -(-nz // bs)
    out = np.empty(gx * gy * gz, np.uint8)
    load().oracle_occupancy(_p(np.ascontiguousarray(dens, np.float32)), nx, ny, nz, bs, halo, threshold, _p(out))
    return out


def env_pyramid(rgba: np.ndarray, levels: int = 12) -> np.ndarray:
    h, w, _ = rgba.shape
    total = sum((1 << (levels - l)) ** 2 for l in range(levels))
    out = np.empty(total, np.float32)
    load().oracle_env_pyramid(_p(np.ascontiguousarray(rgba, np.float32)), w, h, levels, _p(out))
    return out


def svgf_frame(noisy, normal, depth, fwidth, motion, history, z_threshold, normal_threshold, iterations):
    """One SVGF frame on prepared maps (noisy / normal [h, w, 4], depth / fwidth [h, w], motion [h, w, 2]);
    history: dict of color [h,w,4], moments [h,w,4], normal [h,w,4], depth [h,w] (float32, updated in
    place).  Returns the filtered rgba [h, w, 4]."""
    h, w = depth.shape
    arrs = [np.ascontiguousarray(a, np.float32) for a in (noisy, normal, depth, fwidth, motion)]
    for k in ("color", "moments", "normal", "depth"):
        assert history[k].dtype == np.float32 and history[k].flags["C_CONTIGUOUS"]
    out = np.zeros((h, w, 4), np.float32)
    load().oracle_svgf_frame(*[_p(a) for a in arrs], _p(history["color"]), _p(history["moments"]),
                             _p(history["normal"]), _p(history["depth"]), w, h, z_threshold, normal_threshold,
                             iterations, _p(out))
    return out


def eaw(color, pos, nrm, iterations, phi_c=5.0, phi_p=0.1, phi_n=0.1, quirk=0):
    h, w, _ = color.shape
    out = np.empty_like(color)
    load().oracle_eaw(_p(color), _p(pos), _p(nrm), w, h, iterations, phi_c, phi_p, phi_n, quirk, _p(out))
    return out


def rng_stream(seed: int, n: int):
    out = np.empty(n, np.float32)
    st = np.empty(4, np.uint32)
    load().oracle_rng_stream(seed, n, _p(out), _p(st))
    return out, st


class Scene:
    """Holds an OracleScene plus the numpy buffers it points to."""

    def __init__(self, **kw):
        self.s = OracleScene()
        self._keep = {}
        for k, v in kw.items():
            self.set(k, v)

    def set(self, k, v):
        if k in ("density", "sv_data", "occupancy", "env_rgba", "env_pyramid", "nanovdb", "emission", "tf",
                 "sv_local", "iso_grad"):
            arr = None if v is None else np.ascontiguousarray(v)
            self._keep[k] = arr
            setattr(self.s, k, None if arr is None else arr.ctypes.data_as(c_void_p).value)
        elif isinstance(v, (list, tuple, np.ndarray)):
            arr = getattr(self.s, k)
            for i, x in enumerate(v):
                arr[i] = float(x)
        else:
            setattr(self.s, k, v)

    def render(self, threads=0, with_sq=False):
        n = self.s.width * self.s.height * 3
        film = np.zeros(n, np.float64)
        sq = np.zeros(n, np.float64) if with_sq else None
        lk = c_uint64(0)
        _ok(load().oracle_render(ctypes.byref(self.s), _p(film), _p(sq), ctypes.byref(lk), threads))
        return film, sq, lk.value

    def render_rows(self, row0, row1, threads=0):
        film = np.zeros(self.s.width * self.s.height * 3, np.float64)
        lk = c_uint64(0)
        _ok(load().oracle_render_rows(ctypes.byref(self.s), row0, row1, _p(film), ctypes.byref(lk), threads))
        return film, lk.value

    def trace_paths(self, xs, ys, frames, threads=0):
        xs = np.ascontiguousarray(xs, np.int32)
        ys = np.ascontiguousarray(ys, np.int32)
        fr = np.ascontiguousarray(frames, np.uint32)
        out = np.empty((xs.size, 3), np.float32)
        _ok(load().oracle_trace_paths(ctypes.byref(self.s), _p(xs), _p(ys), _p(fr), xs.size, _p(out), threads))
        return out


class double_rounded_math:
    """Context manager: the oracle's transcendentals in double precision rounded to float (the mode
    of the CUDA core's libvpt_b200_dr.so) inside the block."""

    def __init__(self, on: bool = True):
        self.on = on

    def __enter__(self):
        load().oracle_set_double_rounded_math(1 if self.on else 0)
        return self

    def __exit__(self, *exc):
        load().oracle_set_double_rounded_math(0)
        return False


def nanovdb_query(buf: np.ndarray, ijk: np.ndarray):
    """The oracle's restatement of PNanoVDB's accessor: value, dim, active at each voxel."""
    c = np.ascontiguousarray(ijk, np.int32).reshape(-1, 3)
    n = c.shape[0]
    val = np.empty(n, np.float32)
    dim = np.empty(n, np.uint32)
    act = np.empty(n, np.uint8)
    load().oracle_nanovdb_query(_p(buf), n, _p(c), _p(val), _p(dim), _p(act))
    return val, dim, act


def nanovdb_hdda_walk(buf: np.ndarray, origin, direction, lowest_level: int = 8, max_visits: int = 4096):
    o = np.asarray(origin, np.float32)
    d = np.asarray(direction, np.float32)
    vox = np.zeros((max_visits, 3), np.int32)
    dim = np.zeros(max_visits, np.int32)
    act = np.zeros(max_visits, np.uint8)
    lvl = np.zeros(max_visits, np.int32)
    box = np.zeros((max_visits, 6), np.float32)
    t = np.zeros((max_visits, 3), np.float32)
    n = load().oracle_nanovdb_hdda_walk(_p(buf), _p(o), _p(d), lowest_level, max_visits, _p(vox), _p(dim), _p(act),
                                        _p(lvl), _p(box), _p(t))
    if n < 0:
        return None
    return dict(voxel=vox[:n], dim=dim[:n], active=act[:n], level=lvl[:n], box=box[:n], t=t[:n])


# ---- kernel-predicting denoiser (modules/kpn_module/src/Kernel.cu + the libtorch ops around it) ----

def _f(a):
    return np.ascontiguousarray(a, np.float32)


def softmax_channels(x):
    x = _f(x)
    out = np.empty_like(x)
    n, k, h, w = x.shape
    load().oracle_softmax_channels(_p(x), n, k, h, w, _p(out))
    return out


def kpn_apply(image, weights, k, softmax=False):
    image, weights = _f(image), _f(weights)
    if softmax:
        weights = softmax_channels(weights)
    n, c, h, w = image.shape
    wh, ww = weights.shape[2:]
    out = np.zeros((n, c, min(h, wh), min(w, ww)), np.float32)
    load().oracle_kpn_apply(_p(image), _p(weights), n, c, h, w, wh, ww, k, _p(out))
    return out


def kpn_inv_iter(x_hi, pred_lo, x_lo, prev, fused, k, use_prev):
    """inv_iter_kernel (PyTorchDenoiser.cpp:174-179): base image, softmax of the first k*k fused
    channels, per-pixel kernel."""
    x_hi, pred_lo, x_lo, fused = _f(x_hi), _f(pred_lo), _f(x_lo), _f(fused)
    prev = _f(prev) if prev is not None else np.zeros_like(x_hi)
    n, c, h, w = x_hi.shape
    lh, lw = x_lo.shape[2:]
    wh, ww = fused.shape[2:]
    base = np.zeros((n, c, min(h, wh), min(w, ww)), np.float32)
    load().oracle_kpn_inv_iter_base(_p(x_hi), _p(pred_lo), _p(x_lo), _p(prev), _p(fused), n, c, h, w, lh, lw, wh, ww,
                                    k, 1 if use_prev else 0, _p(base))
    return kpn_apply(base, np.ascontiguousarray(fused[:, :k * k]), k, softmax=True)


def avg_pool2(x):
    x = _f(x)
    n, c, h, w = x.shape
    out = np.empty((n, c, h // 2, w // 2), np.float32)
    load().oracle_avg_pool2(_p(x), n * c, h, w, _p(out))
    return out


def grid_sample(prev, uv):
    prev, uv = _f(prev), _f(uv)
    n, c, ph, pw = prev.shape
    h, w = uv.shape[2:]
    out = np.empty((n, c, h, w), np.float32)
    load().oracle_grid_sample(_p(prev), _p(uv), n, c, ph, pw, h, w, _p(out))
    return out
