"""Generates tests/golden/image_filters.npz from the reference's own image compute shaders run on the CPU
(oracle/_ref/libref_image.so, built by oracle/ref_build.py from Data/Shaders/VPT/OctahedralMapper.glsl and
the compute stage of Data/Shaders/Denoiser/EAWDenoise.glsl).

* ``octa_<name>``: the octahedral max-brightness map (level 0 of the importance pyramid) of an
  equirectangular RGBA environment image;
* ``eaw_<name>_<iterations>``: the EAW a-trous chain of the compute path (colour weight exp(-1/phi_c),
  EAWDenoise.glsl:269) with phi = (5, 0.1, 0.1), colour, position and normal weights on.

Run in a container that has the reference tree:  python tests/golden/make_image_golden.py
"""
import ctypes
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import ref_build  # noqa: E402

P = ctypes.c_void_p
PHI = (5.0, 0.1, 0.1)


def env_images():
    rng = np.random.default_rng(9)
    a = np.ones((32, 64, 4), np.float32)
    a[..., :3] = 0.2 + rng.random((32, 64, 3)).astype(np.float32) * 0.05
    a[5:8, 20:24, :3] = 40.0
    b = np.ones((48, 96, 4), np.float32)
    b[..., :3] = rng.random((48, 96, 3)).astype(np.float32) * 3.0
    return {"sunpatch": (a, 64), "noise": (b, 128)}


def eaw_inputs():
    rng = np.random.default_rng(5)
    out = {}
    for name, (h, w) in (("48x64", (48, 64)), ("37x50", (37, 50))):
        color = rng.random((h, w, 4)).astype(np.float32)
        pos = (rng.random((h, w, 4)) * 0.2).astype(np.float32)
        nrm = rng.random((h, w, 4)).astype(np.float32)
        out[name] = (color, pos, nrm)
    return out


def main():
    ref_build.build()
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_image.so"))
    data, meta = {}, {}
    for name, (rgba, res) in env_images().items():
        out = np.zeros(res * res, np.float32)
        assert lib.ref_octahedral_map(rgba.ctypes.data_as(P), rgba.shape[1], rgba.shape[0], res,
                                      out.ctypes.data_as(P)) == 0
        data[f"octa_{name}__env"] = rgba
        data[f"octa_{name}__map"] = out.reshape(res, res)
        meta[f"octa_{name}"] = {"res": res}
        print("octa", name, float(out.max()))
    for name, (color, pos, nrm) in eaw_inputs().items():
        h, w = color.shape[:2]
        data[f"eaw_{name}__color"], data[f"eaw_{name}__position"], data[f"eaw_{name}__normal"] = color, pos, nrm
        for it in (1, 3, 5):
            out = np.zeros_like(color)
            assert lib.ref_eaw_compute(color.ctypes.data_as(P), pos.ctypes.data_as(P), nrm.ctypes.data_as(P), w, h, it,
                                       ctypes.c_float(PHI[0]), ctypes.c_float(PHI[1]), ctypes.c_float(PHI[2]),
                                       out.ctypes.data_as(P)) == 0
            data[f"eaw_{name}_{it}__out"] = out
            meta[f"eaw_{name}_{it}"] = {"input": f"eaw_{name}", "iterations": it, "phi": list(PHI)}
            print("eaw", name, it, float(out.mean()))
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "image_filters.npz")
    np.savez_compressed(path, meta=json.dumps(meta), **data)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
