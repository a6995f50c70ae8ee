"""Sparse (NanoVDB) volumes on the CUDA core, through the C ABI.

* accessor: the core's brick-table volume, loaded from the reference-built NanoVDB buffers
  (tests/golden/sparse_grids.npz) or built by the core itself from the dense grid (GridBuilder
  semantics), returns bit for bit the value, dim and active state the reference's PNanoVDB accessor
  returns at every fixture voxel;
* paths: every camera path of a 1-spp frame on a sparse grid (delta, ratio, NEE, HDDA decomposition
  tracking; nearest / stochastic / trilinear lookups; fp32 and fp16 leaves) against the CPU oracle
  reading the reference-built buffer through its own PNanoVDB restatement.  With the ``dr`` build
  (transcendentals rounded from double on both sides) every path must agree.
"""
import ctypes

import numpy as np
import pytest
import torch

from cloudrendering_b200._lib import VptSparseInfo
from oracle import bridge
from tests.harness import (SPARSE_GRIDS, Core, SceneSpec, gpu_render, oracle_scene, path_agreement, setup_core,
                           sparse_golden, sparse_grid)

pytestmark = pytest.mark.gpu

GOLD = sparse_golden()
CUBE_GRIDS = ["fbm24", "block8b", "saturated40", "tiles256"]  # voxel size 1/n and origin -0.5 on every axis


@pytest.fixture(scope="module")
def core():
    c = Core(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def core_dr():
    c = Core(0, "dr")
    yield c
    c.close()


def dptr(t):
    return ctypes.c_void_p(t.data_ptr())


def query(core, ijk):
    d_ijk = torch.from_numpy(np.ascontiguousarray(ijk, np.int32)).cuda()
    n = ijk.shape[0]
    val = torch.empty(n, dtype=torch.float32, device="cuda")
    dim = torch.empty(n, dtype=torch.int32, device="cuda")
    act = torch.empty(n, dtype=torch.uint8, device="cuda")
    core("vpt_sparse_query", dptr(d_ijk), n, dptr(val), dptr(dim), dptr(act), None)
    torch.cuda.synchronize()
    return val.cpu().numpy(), dim.cpu().numpy().view(np.uint32), act.cpu().numpy()


def info(core):
    i = VptSparseInfo()
    core("vpt_get_sparse_grid_info", ctypes.byref(i))
    return i


def load_nanovdb(core, buf, fp16=False):
    core("vpt_set_option", b"sparse_fp16", 1.0 if fp16 else 0.0)
    core("vpt_set_nanovdb_grid", buf.ctypes.data_as(ctypes.c_void_p), buf.nbytes, 0)


def load_dense_as_sparse(core, name, fp16=False):
    g = np.ascontiguousarray(sparse_grid(name), np.float32)
    nz, ny, nx = g.shape
    core("vpt_set_max_grid_extent", 0.5)
    core("vpt_set_dense_grid", g.ctypes.data_as(ctypes.c_void_p), nx, ny, nz, 0)
    core("vpt_set_option", b"sparse_fp16", 1.0 if fp16 else 0.0)
    core("vpt_set_use_sparse_grid", 1)


def check_accessor(core, g):
    val, dim, act = query(core, g["ijk"])
    assert np.array_equal(val.view(np.uint32), g["value"].view(np.uint32))
    assert np.array_equal(dim, g["dim"])
    assert np.array_equal(act, g["active"])


@pytest.mark.parametrize("name", SPARSE_GRIDS)
def test_nanovdb_buffer_accessor_bit_exact(core, name):
    g = GOLD[name]
    load_nanovdb(core, g["buf"])
    check_accessor(core, g)
    i = info(core)
    ib = g["meta"]["index_bbox"]
    assert list(i.root_min) == ib[:3] and list(i.root_max) == ib[3:]
    assert list(i.world_min) == g["meta"]["world_bbox"][:3] and list(i.world_max) == g["meta"]["world_bbox"][3:]


@pytest.mark.parametrize("name", SPARSE_GRIDS)
def test_dense_to_sparse_matches_reference_gridbuilder(core, name):
    """The core's own dense -> sparse build gives the tree the reference's GridBuilder gives."""
    g = GOLD[name]
    load_dense_as_sparse(core, name)
    check_accessor(core, g)
    i = info(core)
    ib = g["meta"]["index_bbox"]
    assert list(i.root_min) == ib[:3] and list(i.root_max) == ib[3:]
    if name in CUBE_GRIDS:
        assert list(i.world_min) == g["meta"]["world_bbox"][:3]
        assert list(i.world_max) == g["meta"]["world_bbox"][3:]
    core("vpt_set_use_sparse_grid", 0)


def scene(name, **kw):
    base = dict(grid=sparse_grid(name), extinction=120.0, albedo=0.99, g=0.85, width=48, height=48, env="default",
                linear_rgb=1, cam_pos=(0.3, 0.4, 1.4), max_grid_extent=0.5, max_bounces=64)
    base.update(kw)
    return SceneSpec(**base)


def sparse_oracle(core, sp, g, fp16=False):
    """Oracle scene on the reference-built buffer, with the core's camera and sparse render box."""
    i = info(core)
    sc = oracle_scene(core, sp, 1)
    wb = g["meta"]["world_bbox"]
    sc.set("box_min", list(i.box_min))
    sc.set("box_max", list(i.box_max))
    sc.set("grid_min", [float(np.float32(v)) for v in wb[:3]])
    sc.set("grid_max", [float(np.float32(v)) for v in wb[3:]])
    sc.set("nanovdb", g["buf"])
    sc.set("sparse_lowest_level", int(i.lowest_level))
    sc.set("sparse_fp16", 1 if fp16 else 0)
    return sc


PATH_CASES = {
    "delta_stochastic": dict(mode="delta"),
    "delta_nearest": dict(mode="delta", interp="nearest"),
    "delta_trilinear": dict(mode="delta", interp="trilinear"),
    "ratio": dict(mode="ratio"),
    "nee": dict(mode="nee"),
    "decomposition": dict(mode="decomposition"),
    "decomposition_nearest": dict(mode="decomposition", interp="nearest"),
    "decomposition_trilinear_uncapped": dict(mode="decomposition", interp="trilinear", max_bounces=0),
}


@pytest.mark.parametrize("grid", ["fbm24", "saturated40"])
@pytest.mark.parametrize("case", sorted(PATH_CASES))
@pytest.mark.parametrize("variant", ["default", "dr"])
@pytest.mark.parametrize("source", ["nanovdb", "dense"])
def test_sparse_path_parity(core, core_dr, grid, case, variant, source):
    c = core if variant == "default" else core_dr
    g = GOLD[grid]
    sp = scene(grid, **PATH_CASES[case])
    setup_core(c, sp)
    if source == "nanovdb":
        load_nanovdb(c, g["buf"])
    else:
        c("vpt_set_use_sparse_grid", 1)
    s, _ = gpu_render(c, sp, 1, stats=False)
    sc = sparse_oracle(c, sp, g)
    ys, xs = np.mgrid[0:sp.height, 0:sp.width]
    with bridge.double_rounded_math(variant == "dr"):
        ref = sc.trace_paths(xs.reshape(-1), ys.reshape(-1), np.zeros(xs.size, np.uint32)).reshape(
            sp.height, sp.width, 3)
    if source == "dense":
        c("vpt_set_use_sparse_grid", 0)
    agree = path_agreement(s.astype(np.float32), ref)
    lit = float(np.mean(ref.sum(axis=-1) > 0))
    print(f"[{variant}/{source}] {grid} {case}: path agreement {agree:.5f} (non-black paths {lit:.2f})")
    assert agree >= (0.99 if variant == "default" else 0.999)


@pytest.mark.parametrize("case", ["delta_stochastic", "decomposition"])
def test_sparse_fp16_leaves_path_parity(core_dr, case):
    g = GOLD["saturated40"]
    sp = scene("saturated40", **PATH_CASES[case])
    setup_core(core_dr, sp)
    load_nanovdb(core_dr, g["buf"], fp16=True)
    assert info(core_dr).fp16 == 1
    s, _ = gpu_render(core_dr, sp, 1, stats=False)
    sc = sparse_oracle(core_dr, sp, g, fp16=True)
    ys, xs = np.mgrid[0:sp.height, 0:sp.width]
    with bridge.double_rounded_math(True):
        ref = sc.trace_paths(xs.reshape(-1), ys.reshape(-1), np.zeros(xs.size, np.uint32)).reshape(
            sp.height, sp.width, 3)
    core_dr("vpt_set_option", b"sparse_fp16", 0.0)
    agree = path_agreement(s.astype(np.float32), ref)
    print(f"fp16 {case}: path agreement {agree:.5f}")
    assert agree >= 0.999


def test_sparse_rejects_dense_only_trackers(core):
    load_dense_as_sparse(core, "fbm24")
    core("vpt_set_vpt_mode", 4)  # residual ratio tracking
    core("vpt_set_resolution", 8, 8)
    st = core.lib.vpt_render_frames(core.ctx, 1, None)
    assert st == 6  # VPT_ERR_UNSUPPORTED, as in the reference (dense only)
    core("vpt_set_vpt_mode", 0)
    core("vpt_set_use_sparse_grid", 0)
