"""Generates tests/golden/supervoxel_grids.npz from the reference's own supervoxel grid builders
(src/PathTracer/SuperVoxelGrid.cpp with src/DensityField.cpp, compiled unmodified for the CPU by
oracle/ref_build.py into oracle/_ref/libref_supervoxel.so).

For every raw (un-normalised) grid and interpolation it stores what the reference uploads to its
supervoxel textures: SuperVoxelGridDecompositionTracking's (min, max) pairs and occupancy, and
SuperVoxelGridResidualRatioTracking's (mu_c, mu_r_bar) pairs (setExtinction(700)) and occupancy, with
clampToZeroBorder on (the pass's default).

Run in a container that has the reference tree:  python tests/golden/make_supervoxel_golden.py
"""
import ctypes
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import bridge, ref_build  # noqa: E402

EXTINCTION = 700.0


def grids():
    out = {}
    g = bridge.fbm((40, 24, 33), 7, base_frequency=3.0, contrast=3.5)
    out["fbm_ragged"] = (g * np.float32(3.0) + np.float32(0.5)).astype(np.float32)  # min > 0: normalisation
    out["fbm64"] = bridge.fbm(64, 11, base_frequency=3.0, contrast=3.5)
    b = np.zeros((8, 8, 8), np.float32)
    b[1:7, 1:7, 1:7] = 1.0
    out["block8_boundary"] = b
    out["constant"] = np.full((16, 12, 20), 0.8, np.float32)  # min == max: DensityField uses min = 0
    out["tiny6"] = bridge.fbm(6, 3, base_frequency=2.0, contrast=3.5)  # supervoxel size halves to 2
    return out


def main():
    ref_build.build()
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_supervoxel.so"))
    P = ctypes.c_void_p
    data, meta = {}, {}
    for name, raw in grids().items():
        nz, ny, nx = raw.shape
        data[name + "__raw"] = raw
        for interp in (0, 1):
            key = f"{name}__i{interp}"
            dims = (ctypes.c_int * 4)()
            n_max = nx * ny * nz
            mm = np.zeros(2 * n_max, np.float32)
            occ = np.zeros(n_max, np.uint8)
            assert lib.ref_supervoxel_decomposition(raw.ctypes.data_as(P), nx, ny, nz, 8, interp, 1,
                                                    mm.ctypes.data_as(P), occ.ctypes.data_as(P), dims) == 0
            n = dims[0] * dims[1] * dims[2]
            data[key + "__minmax"] = mm[:2 * n].copy()
            data[key + "__occ_decomposition"] = occ[:n].copy()
            pairs = np.zeros(2 * n_max, np.float32)
            assert lib.ref_supervoxel_rrt(raw.ctypes.data_as(P), nx, ny, nz, 8, interp, 1,
                                          ctypes.c_float(EXTINCTION), pairs.ctypes.data_as(P), occ.ctypes.data_as(P),
                                          dims) == 0
            data[key + "__rrt"] = pairs[:2 * n].copy()
            data[key + "__occ_rrt"] = occ[:n].copy()
            meta[key] = {"grid": name, "interp": interp, "dims": list(dims), "extinction": EXTINCTION}
            print(key, list(dims), float(data[key + "__minmax"][1::2].mean()))
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "supervoxel_grids.npz")
    np.savez_compressed(out, meta=json.dumps(meta), **data)
    print("wrote", out, os.path.getsize(out), "bytes")


if __name__ == "__main__":
    main()
