"""ctypes bridge to the reference's NanoVDB code compiled for the CPU (TEST INFRASTRUCTURE ONLY):
``oracle/_ref/libref_nanovdb_builder.so`` (the vendored GridBuilder, driven as
CloudData::getSparseDensityField drives it) and ``oracle/_ref/libref_pnanovdb.so`` (PNanoVDB.glsl in
its C mode: read accessor, map, HDDA).  Both are built by oracle/ref_build.py."""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_double, c_float, c_int, c_int32, c_uint8, c_uint32, c_uint64, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILDER = os.path.join(HERE, "_ref", "libref_nanovdb_builder.so")
PNANOVDB = os.path.join(HERE, "_ref", "libref_pnanovdb.so")

_b = None
_p = None


def available() -> bool:
    return os.path.exists(BUILDER) and os.path.exists(PNANOVDB)


def _builder():
    global _b
    if _b is None:
        lib = ctypes.CDLL(BUILDER)
        lib.refvdb_build_from_dense.restype = c_int
        lib.refvdb_build_from_dense.argtypes = [c_void_p, c_int, c_int, c_int, c_double, c_double, c_double, c_double,
                                                POINTER(c_void_p), POINTER(c_uint64)]
        lib.refvdb_free.argtypes = [c_void_p]
        lib.refvdb_grid_info.restype = c_int
        lib.refvdb_grid_info.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p]
        _b = lib
    return _b


def _pn():
    global _p
    if _p is None:
        lib = ctypes.CDLL(PNANOVDB)
        lib.refvdb_query.argtypes = [c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p]
        lib.refvdb_map.argtypes = [c_void_p, c_int, c_int, c_void_p, c_void_p]
        lib.refvdb_root_bbox.argtypes = [c_void_p, c_void_p]
        lib.refvdb_hdda_walk.restype = c_int
        lib.refvdb_hdda_walk.argtypes = [c_void_p, c_void_p, c_void_p, c_int, c_int, c_void_p, c_void_p, c_void_p,
                                         c_void_p, c_void_p, c_void_p]
        _p = lib
    return _p


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(c_void_p)


def build_from_dense(dense: np.ndarray, dx: float, origin) -> np.ndarray:
    """NanoVDB float grid (bytes as a uint32 array) from a dense [nz, ny, nx] grid of normalised
    densities, as CloudData::getSparseDensityField builds it."""
    d = np.ascontiguousarray(dense, np.float32)
    nz, ny, nx = d.shape
    out = c_void_p()
    size = c_uint64()
    st = _builder().refvdb_build_from_dense(_ptr(d), nx, ny, nz, float(dx), float(origin[0]), float(origin[1]),
                                            float(origin[2]), ctypes.byref(out), ctypes.byref(size))
    if st != 0:
        raise RuntimeError("GridBuilder failed")
    n = size.value
    buf = np.empty((n + 3) // 4, np.uint32)
    ctypes.memmove(buf.ctypes.data, out, n)
    _builder().refvdb_free(out)
    return buf


def grid_info(buf: np.ndarray):
    wb = np.zeros(6, np.float64)
    ib = np.zeros(6, np.int32)
    vs = np.zeros(3, np.float64)
    if _builder().refvdb_grid_info(_ptr(buf), _ptr(wb), _ptr(ib), _ptr(vs)) != 0:
        raise RuntimeError("invalid grid")
    return wb, ib, vs


def query(buf: np.ndarray, ijk: np.ndarray):
    c = np.ascontiguousarray(ijk, np.int32).reshape(-1, 3)
    n = c.shape[0]
    val = np.empty(n, np.float32)
    dim = np.empty(n, np.uint32)
    act = np.empty(n, np.uint8)
    _pn().refvdb_query(_ptr(buf), n, _ptr(c), _ptr(val), _ptr(dim), _ptr(act))
    return val, dim, act


def map_points(buf: np.ndarray, pts: np.ndarray, which: int) -> np.ndarray:
    """which: 0 world->index, 1 world->index direction, 2 index->world (float, as the shader)."""
    p = np.ascontiguousarray(pts, np.float32).reshape(-1, 3)
    out = np.empty_like(p)
    _pn().refvdb_map(_ptr(buf), p.shape[0], which, _ptr(p), _ptr(out))
    return out


def root_bbox(buf: np.ndarray) -> np.ndarray:
    out = np.zeros(6, np.int32)
    _pn().refvdb_root_bbox(_ptr(buf), _ptr(out))
    return out


def hdda_walk(buf: np.ndarray, origin, direction, lowest_level: int = 8, max_visits: int = 4096):
    o = np.asarray(origin, np.float32)
    d = np.asarray(direction, np.float32)
    vox = np.zeros((max_visits, 3), np.int32)
    dim = np.zeros(max_visits, np.int32)
    act = np.zeros(max_visits, np.uint8)
    lvl = np.zeros(max_visits, np.int32)
    box = np.zeros((max_visits, 6), np.float32)
    t = np.zeros((max_visits, 3), np.float32)
    n = _pn().refvdb_hdda_walk(_ptr(buf), _ptr(o), _ptr(d), lowest_level, max_visits, _ptr(vox), _ptr(dim), _ptr(act),
                               _ptr(lvl), _ptr(box), _ptr(t))
    if n < 0:
        return None
    return dict(voxel=vox[:n], dim=dim[:n], active=act[:n], level=lvl[:n], box=box[:n], t=t[:n])
